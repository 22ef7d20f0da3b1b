// The C-ABI (include/coral_b200.h): a handle owns the parsed problem, the
// device-resident state, operators, LU factors and transform buffers, one CUDA
// stream and a CUDA graph of one timestep.
#include <algorithm>
#include <cmath>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <thread>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sys/stat.h>
#include <cerrno>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/coral_b200.h"
#include "device.hpp"
#include "host.hpp"

using namespace coral;

namespace coral {
ClosureImpl* closure_impl(coral_closure* c);  // closure.cu
}

namespace {

thread_local std::string g_create_error;

#define CK(call)                                                                                   \
  do {                                                                                             \
    cudaError_t e_ = (call);                                                                       \
    if (e_ != cudaSuccess)                                                                         \
      throw CoralError(e_ == cudaErrorMemoryAllocation ? CORAL_ENOMEM : CORAL_ECUDA,               \
                       std::string(#call) + ": " + cudaGetErrorString(e_));                       \
  } while (0)

struct DevAlloc {
  std::vector<void*> ptrs;
  size_t bytes = 0;
  template <typename T>
  T* get(size_t n) {
    if (n == 0) n = 1;
    void* p = nullptr;
    cudaError_t e = cudaMalloc(&p, n * sizeof(T));
    if (e != cudaSuccess)
      throw CoralError(CORAL_ENOMEM, "device allocation of " + std::to_string(n * sizeof(T)) + " bytes failed: " +
                                         cudaGetErrorString(e));
    ptrs.push_back(p);
    bytes += n * sizeof(T);
    return static_cast<T*>(p);
  }
  template <typename T>
  T* upload(const std::vector<T>& v) {
    T* p = get<T>(v.size());
    if (!v.empty()) CK(cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
    return p;
  }
  void free_all() {
    for (void* p : ptrs) cudaFree(p);
    ptrs.clear();
  }
};

bool smooth23(int n) {
  if (n <= 0) return false;
  while (n % 2 == 0) n /= 2;
  while (n % 3 == 0) n /= 3;
  return n == 1;
}

struct KSys {
  SystemOps ops;
  DevEll M, L, NL;
  int T, kl, ku, ldab;
  double2 *field, *aux;
  double2* Kstd[kMaxStages];
  double2* Khat[kMaxStages];
  double2* ab;           // complex LAPACK-band factors (general recipes)
  double* abr;           // real-scaled factors (recipes that admit the +-i scaling)
  bool real = false;
  unsigned char *rowflip = nullptr, *colflip = nullptr;
  unsigned char* dpiv;
  int* info;
  // class split of the real-scaled solve (SystemOps::ncls == 2); when unsplit:
  // ncls = 1, Tc = T, the band (kl_s, ku_s, ldab_s) of the whole system, work = aux
  int ncls = 1, Tc = 0, kl_s = 0, ku_s = 0, ldab_s = 0, wst = 0;
  int *row_pos = nullptr, *col_pos = nullptr, *cls_row = nullptr, *cls_col = nullptr;
  unsigned char* colflip_cls = nullptr;
  DevEll Lp;
  // per class column, band entries nonzero in any block (thread-per-block layout)
  unsigned long long* cmask = nullptr;
  unsigned *lmask = nullptr, *umask = nullptr;
  // operator-stationary K_std: tile windows and window-relative L
  int* tile_win = nullptr;
  int tile_lwin_max = 0;
  DevGEll Lw;
  int* rhs_win = nullptr;
  int rhs_win_max = 0;
  DevEll Mw, NLw;
  DevGEll NLg;
  double2* work = nullptr;
  double2* work2 = nullptr;  // thread-per-block layout of the active systems' vectors (split only)
  std::vector<std::vector<int>> tab_t;   // per var: [NZ][kTabW]
  std::vector<std::vector<double>> tab_v;
  std::vector<int*> d_tab_t;
  std::vector<double*> d_tab_v;
  std::vector<int*> d_var_pos;
  std::vector<int*> d_sq_col;
  std::vector<double*> d_sq_val;
};

struct ZSys {
  SystemOps ops;
  ZeroSysDev dev;
  std::vector<std::vector<int>> tab_t;
  std::vector<std::vector<double>> tab_v;
  std::vector<int*> d_tab_t;
  std::vector<double*> d_tab_v;
};

}  // namespace

namespace coral {
void set_global_error(const std::string& msg) { g_create_error = msg; }
}  // namespace coral

// side streams of the y-chunked pipeline of a stage (inverse x, fused z and
// forward x passes per band of y rows, bands round-robin over the streams)
constexpr int kYStreams = 3;

// Output files written behind the time step (the reference writes them
// synchronously, PL_IMEX_timestepping_output.f90:489-578): an object formed on
// the device is copied into a page-locked staging buffer on a copy stream, and a
// host thread writes the file once that copy has completed, while the next
// steps run.  At most kOutBufs staging buffers (each grown to the largest
// object) are in flight; flush() waits for every file and reports the first
// failed write.
struct OutputWriter {
  static constexpr int kOutBufs = 2;
  struct Job {
    cudaEvent_t done;
    int buf;
    size_t n;
    std::string dir, path;
  };
  int device = 0;
  cudaStream_t copy = nullptr;
  double* pin[kOutBufs] = {};
  size_t cap[kOutBufs] = {};
  bool busy[kOutBufs] = {};
  cudaEvent_t last = nullptr;  // the latest copy out of the device buffer
  std::mutex mu;
  std::condition_variable cv;
  std::deque<Job> q;
  std::thread th;
  bool stop = false;
  int pending = 0;
  std::string err;

  void start(int dev) {
    device = dev;
    if (th.joinable()) return;
    th = std::thread([this] { run(); });
  }
  void run() {
    cudaSetDevice(device);
    for (;;) {
      Job j;
      {
        std::unique_lock<std::mutex> lk(mu);
        cv.wait(lk, [&] { return stop || !q.empty(); });
        if (q.empty()) return;
        j = q.front();
        q.pop_front();
      }
      std::string e;
      if (cudaEventSynchronize(j.done) != cudaSuccess) e = "copy of " + j.path + " failed";
      if (e.empty() && mkdir_all(j.dir) != 0) e = "cannot create " + j.dir;
      if (e.empty()) {
        FILE* fp = std::fopen(j.path.c_str(), "wb");
        if (!fp) {
          e = "cannot open " + j.path;
        } else {
          if (std::fwrite(pin[j.buf], sizeof(double), j.n, fp) != j.n) e = "short write in " + j.path;
          std::fclose(fp);
        }
      }
      cudaEventDestroy(j.done);
      std::lock_guard<std::mutex> lk(mu);
      if (!e.empty() && err.empty()) err = e;
      busy[j.buf] = false;
      --pending;
      cv.notify_all();
    }
  }
  static int mkdir_all(const std::string& d) {
    std::string cur;
    for (size_t i = 0; i <= d.size(); ++i) {
      if ((i == d.size() || d[i] == '/') && !cur.empty() && mkdir(cur.c_str(), 0755) != 0 && errno != EEXIST)
        return -1;
      if (i < d.size()) cur.push_back(d[i]);
    }
    return 0;
  }
  // copy n doubles of the device buffer src (formed on stream s) out and queue
  // the file
  void submit(const double* src, size_t n, cudaStream_t s, const std::string& dir, const std::string& path) {
    int b = -1;
    {
      std::unique_lock<std::mutex> lk(mu);
      cv.wait(lk, [&] {
        for (int i = 0; i < kOutBufs; ++i)
          if (!busy[i]) return true;
        return false;
      });
      for (int i = 0; i < kOutBufs && b < 0; ++i)
        if (!busy[i]) b = i;
      busy[b] = true;
    }
    if (cap[b] < n) {
      if (pin[b]) cudaFreeHost(pin[b]);
      pin[b] = nullptr;
      cap[b] = 0;
      if (cudaMallocHost(&pin[b], n * sizeof(double)) != cudaSuccess) {
        cudaGetLastError();
        std::lock_guard<std::mutex> lk(mu);
        busy[b] = false;
        throw CoralError(CORAL_ENOMEM, "page-locked output buffer");
      }
      cap[b] = n;
    }
    if (!copy) CK(cudaStreamCreateWithFlags(&copy, cudaStreamNonBlocking));
    if (!last) CK(cudaEventCreateWithFlags(&last, cudaEventDisableTiming));
    cudaEvent_t formed, done;
    CK(cudaEventCreateWithFlags(&formed, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&done, cudaEventDisableTiming));
    CK(cudaEventRecord(formed, s));
    CK(cudaStreamWaitEvent(copy, formed, 0));
    CK(cudaMemcpyAsync(pin[b], src, n * sizeof(double), cudaMemcpyDeviceToHost, copy));
    CK(cudaEventRecord(done, copy));
    CK(cudaEventRecord(last, copy));
    cudaEventDestroy(formed);
    std::lock_guard<std::mutex> lk(mu);
    q.push_back(Job{done, b, n, dir, path});
    ++pending;
    cv.notify_all();
  }
  // stream s waits for the latest copy before it writes the device buffer again
  void order(cudaStream_t s) {
    if (last) CK(cudaStreamWaitEvent(s, last, 0));
  }
  void flush() {
    std::unique_lock<std::mutex> lk(mu);
    cv.wait(lk, [&] { return pending == 0; });
    if (!err.empty()) {
      const std::string e = err;
      err.clear();
      throw CoralError(CORAL_EIO, e);
    }
  }
  ~OutputWriter() {
    {
      std::lock_guard<std::mutex> lk(mu);
      stop = true;
      cv.notify_all();
    }
    if (th.joinable()) th.join();
    for (auto& p : pin)
      if (p) cudaFreeHost(p);
    if (last) cudaEventDestroy(last);
    if (copy) cudaStreamDestroy(copy);
  }
};

struct coral_handle {
  std::string err;
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaStream_t ystream[kYStreams] = {};
  cudaEvent_t yfork = nullptr, yjoin[kYStreams] = {};
  Parameters P;
  Recipe R;
  std::unique_ptr<Geometry> G;
  Tableau TB;
  Dims d;
  DevAlloc mem;
  std::vector<KSys> ks;
  std::vector<ZSys> zs;
  int nF = 0, nQ = 0, nact = 0;
  int* d_act_index = nullptr;
  int* d_act_list = nullptr;
  double *d_kx = nullptr, *d_ky = nullptr, *d_wz = nullptr, *d_wzinv = nullptr;
  FftPlan py{}, px{}, pz{};
  double2* dct_tw = nullptr;
  FullVarDev* d_fv = nullptr;
  bool fv_single = false;  // every full variable: mean terms, then exactly one kxky term
  int* d_tab_id_t = nullptr;
  double* d_tab_id_v = nullptr;
  // z derivatives in full-variable builds: each dz term is built by k_full_dz
  // into its own spectral buffer, which the build reads as pseudo-system
  // ks.size() + j through an identity stencil
  struct DzJob { int set, T, order; const int* tab_t; const double* tab_v; double dsca; double2* out; };
  std::vector<DzJob> dz_jobs;
  // the same for dz terms of mean variables: one profile each, read as mean
  // pseudo-system zs.size() + j
  struct ZDzJob { int set, order; const int* tab_t; const double* tab_v; double dsca; double* out; };
  std::vector<ZDzJob> zdz_jobs;
  QuadDesc quads{};
  std::vector<int> zmean_quads;
  double2 *Y1 = nullptr, *qspec = nullptr, *tmp_spec = nullptr;
  double *Y2 = nullptr, *fphys = nullptr, *tmp_phys = nullptr;
  double* ke_partial = nullptr;
  double* ke_total = nullptr;  // device: total of ke_partial (coral_diagnostics)
  size_t n_ke_partial = 0;
  unsigned long long* cfl_bits = nullptr;
  unsigned int* flags = nullptr;
  int* zinfo = nullptr;
  double dt_factored = -1.0;
  cudaGraphExec_t graph = nullptr;
  double graph_dt = -1.0;
  long long launches = 0;
  int launches_per_step = 0;
  // timeseries objects of coral.timeseries (output_global_quantities,
  // PL_IMEX_timestepping_output.f90:5-231): file name of each object and the
  // per-CTA partial sums / totals on the device
  std::vector<std::string> ts_file;
  double* ts_partial = nullptr;   // [z_fused_ctas][kMaxTs]
  size_t ts_ncta = 0;
  double* ts_out = nullptr;       // [kMaxTs], totals of the last step's first stage
  double* h_pin = nullptr;        // page-locked readback: kMaxTs timeseries values, 4 CFL maxima
  // time keeping of the driver loop (src/misc/timeKeeping.f90:22-49)
  double time = 0.0, dt_current = 0.0, dt_target = 0.0;
  long long i_timestep = 1, refactorizations = 0;
  // timeseries rows not yet written: (i_timestep, time, values)
  std::vector<std::pair<long long, std::vector<double>>> ts_rows;
  // user outputs (coral.usrOutput): kind 0 volume, 1 z slice, 2 y slice, 3 x slice,
  // 4 weighted z sum, 5 profile; src >= 0 a full variable, -1 - q quadratic
  // variable q; index 0-based; the reference's counters and time_integer
  struct UsrOut { int kind, src, index; long long period, counter; };
  std::vector<UsrOut> uo;
  long long time_integer = 1;
  double* uo_buf = nullptr;  // one physical field: an object's file contents before the copy back
  std::unique_ptr<OutputWriter> writer;
  // z transforms: 0 = FP64 FFT (k_z_fused), 1 = int8-digit contractions on the
  // tensor cores (zsplit.cu); form_last = the form of the last step (KE sums)
  int zform = 0, zform_last = 0;
  bool hermitian_kx0 = false;  // project the kx = 0 line onto its Hermitian part after each step
  // the reference's command-line switches (coral_create_with_args)
  bool smagorinsky = false;        // --withHorizontalSmagorinsky
  double smago_prefactor = 1.0;    // --smagorinsky-prefactor
  double cfl_factor_z = 1.0;       // --cflFactor-along-z
  // full variables that are not plain transforms: penalisation fields ([y][x][z]
  // each), the Smagorinsky viscosity profile and the z operations of surface
  // values and vertical decompositions (marching.f90:505-575)
  std::vector<double*> penal_phys;  // per full variable, null unless penalised
  int smago_var = -1;
  std::vector<int> smago_src;       // full variables dxUfull, dyUfull, dxVfull, dyVfull present
  double* smago_prof = nullptr;     // [NZAA], carried from stage to stage
  double* smago_part = nullptr;     // [NYAA][NZAA] scratch
  struct ZFilter { int var, extract, decomp; };
  std::vector<ZFilter> zfilters;
  double* d_zgrid = nullptr;        // Gauss-Chebyshev grid (PL_cheby_misc.f90:19-27)
  // sources of the mean equations: physical profiles on the z grid by index
  // (defaults: the reference's PL_user_sources_definitions.f90) and the constant
  // K_hat terms per mean system on the device
  std::map<int, std::vector<double>> src_phys;
  std::vector<double*> d_src;
  std::string src_missing;          // non-empty: a referenced source has no profile
  // kernel variants chosen by coral_autotune (defaults: the choices measured best at 384^2 x 192)
  struct Tune {
    int x_plan = 1;         // x passes: 1 two-pass FFT plans, 0 three-pass
    int fwd_y_grid = 0;     // forward y pass: 0 persistent pipelined, 1 one CTA per tile
    int generic_tiles = 0;  // operator tile kernels: 0 compiled group layouts, 1 run-time forms
    int subst_rt = 0;       // band substitution: 0 compiled band, 1 run-time band
    int z_batch6 = 1;       // fused z pass: 1 forward batches of 6 lines (3 CTAs per SM), 0 of 9 lines
    int inv_x_tiles = 1;    // inverse x pass: 1 one CTA per tile, 0 persistent pipelined
    int factor_window = 1;  // band factorisation: 1 shared-memory window, 0 in place in global memory
    int inv_y_loop = 0;     // inverse y pass: 0 single-term build where the recipe allows, 1 term loop
    int y_chunks = 1;       // stage passes inverse x -> z -> forward x in this many bands of y rows on
                            // kYStreams streams (grids of at least 288 x 288 points); 1: whole passes
  } tune;
  // learned closure (not owned) and its output [9][y][x][z]
  coral_closure* closure = nullptr;
  double* tau = nullptr;
  unsigned char *zmat_inv = nullptr, *zmat_fwd = nullptr;
  double* ke_partial_split = nullptr;  // [forward CTAs][3]
  size_t n_ke_split = 0;
  double* ts_partial_split = nullptr;  // [inverse + forward CTAs][kMaxTs]
  size_t ts_rows_split = 0, ts_inv_rows = 0;
};

namespace {

FftPlan make_plan(DevAlloc& mem, int N) {
  FftPlan p{};
  p.N = N;
  int n = N, s = 0;
  while (n % 4 == 0) { p.radix[s++] = 4; n /= 4; }
  while (n % 3 == 0) { p.radix[s++] = 3; n /= 3; }
  while (n % 2 == 0) { p.radix[s++] = 2; n /= 2; }
  if (n != 1 || s > 16) throw CoralError(CORAL_EUNSUPPORTED, "transform length " + std::to_string(N) + " is not 2^a 3^b");
  p.nst = s;
  std::vector<double2> tw(N);
  const long double pi = 3.141592653589793238462643383279502884L;
  for (int k = 0; k < N; ++k) {
    long double a = -2.0L * pi * (long double)k / (long double)N;
    tw[k] = make_double2((double)cosl(a), (double)sinl(a));
  }
  p.tw = mem.upload(tw);
  return p;
}

DevEll upload_ell(DevAlloc& mem, const EllOp& op) {
  DevEll e{};
  e.rows = op.rows;
  e.width = op.width;
  e.ngroups = (int)op.groups.size();
  if (e.ngroups > kMaxGroups) throw CoralError(CORAL_EUNSUPPORTED, "too many (kx,ky) monomials in one operator");
  for (int g = 0; g < e.ngroups; ++g) {
    e.gkx[g] = op.groups[g].first;
    e.gky[g] = op.groups[g].second;
  }
  std::vector<int> cg((size_t)op.rows * op.width, 0);
  std::vector<double> val((size_t)op.rows * op.width, 0.0);
  for (int r = 0; r < op.rows; ++r)
    for (int k = 0; k < op.width; ++k) {
      const size_t src = (size_t)r * op.width + k, dst = (size_t)k * op.rows + r;
      if (op.col[src] < 0) continue;
      if (op.col[src] >= (1 << 24)) throw CoralError(CORAL_EUNSUPPORTED, "operator column index too large");
      cg[dst] = op.col[src] | (op.grp[src] << 24);
      val[dst] = op.val[src];
    }
  e.cg = mem.upload(cg);
  e.val = mem.upload(val);
  return e;
}

// The grouped form of an operator for the tile kernels (DevGEll): groups whose
// (column, value) entries coincide in every row are merged (their coefficients
// add), then each row's entries are laid out group by group in fixed slot
// ranges.  Returns valid = 0 when the layout does not fit the register slots.
DevGEll upload_gell(DevAlloc& mem, const EllOp& op) {
  DevGEll e{};
  e.rows = op.rows;
  const int G = (int)op.groups.size();
  // entries of group g in row t, in slot order
  auto entries = [&](int t, int g) {
    std::vector<std::pair<int, double>> v;
    for (int k = 0; k < op.width; ++k) {
      const size_t i = (size_t)t * op.width + k;
      if (op.col[i] >= 0 && op.grp[i] == g) v.emplace_back(op.col[i], op.val[i]);
    }
    return v;
  };
  std::vector<int> cls(G, -1);   // merged group of each monomial group
  std::vector<int> rep;          // representative monomial group of each merged group
  for (int g = 0; g < G; ++g) {
    for (size_t c = 0; c < rep.size() && cls[g] < 0; ++c) {
      bool same = true;
      for (int t = 0; t < op.rows && same; ++t) same = entries(t, g) == entries(t, rep[c]);
      if (same) cls[g] = (int)c;
    }
    if (cls[g] < 0) {
      cls[g] = (int)rep.size();
      rep.push_back(g);
    }
  }
  const int NG = (int)rep.size();
  if (NG > kMaxGroups) return e;
  std::vector<int> wid(NG, 0);
  for (int t = 0; t < op.rows; ++t)
    for (int c = 0; c < NG; ++c) wid[c] = std::max(wid[c], (int)entries(t, rep[c]).size());
  int W = 0;
  for (int c = 0; c < NG; ++c) W += wid[c];
  if (W > kGSlots) return e;
  for (int g = 0; g < G; ++g) {
    const int c = cls[g];
    if (e.nmono[c] >= kGMono) return DevGEll{};
    e.mkx[c][e.nmono[c]] = op.groups[g].first;
    e.mky[c][e.nmono[c]] = op.groups[g].second;
    ++e.nmono[c];
  }
  std::vector<int> col((size_t)W * op.rows, 0);
  std::vector<double> val((size_t)W * op.rows, 0.0);
  int off = 0;
  for (int c = 0; c < NG; ++c) {
    for (int k = 0; k < wid[c]; ++k) e.slot_grp[off + k] = c;
    for (int t = 0; t < op.rows; ++t) {
      const auto v = entries(t, rep[c]);
      for (size_t k = 0; k < v.size(); ++k) {
        col[(size_t)(off + k) * op.rows + t] = v[k].first;
        val[(size_t)(off + k) * op.rows + t] = v[k].second;
      }
    }
    off += wid[c];
  }
  e.width = W;
  e.ngroups = NG;
  e.col = mem.upload(col);
  e.val = mem.upload(val);
  e.valid = 1;
  return e;
}

// Galerkin -> Chebyshev table of one variable: tab[n][k] = (state index, value)
void stencil_tab(const SystemOps& o, int v, int NZ, std::vector<int>& tt, std::vector<double>& tv) {
  tt.assign((size_t)NZ * kTabW, -1);
  tv.assign((size_t)NZ * kTabW, 0.0);
  for (int n = 0; n < NZ; ++n) {
    const auto& row = o.stencil_rows[v][n];
    if ((int)row.size() > kTabW) throw CoralError(CORAL_EUNSUPPORTED, "stencil row wider than the table");
    for (size_t k = 0; k < row.size(); ++k) {
      tt[(size_t)n * kTabW + k] = o.var_pos[v][row[k].first];
      tv[(size_t)n * kTabW + k] = row[k].second;
    }
  }
}

// The two sources of the reference's default PL_user_sources_definitions.f90 on
// the Gauss-Chebyshev grid: source01 = HovEll exp(-z HovEll) / (1 - exp(-HovEll))
// - 1 (HovEll a sourceParam; sourceParams gives 0 when the file has none, which
// makes it NaN, and the reference stops when the file has others but not
// HovEll: source01 then stays undefined), source02 = -1.
void default_sources(coral_handle* h) {
  const Geometry& g = *h->G;
  const double pi = 4.0 * std::atan(1.0);
  std::vector<double> z(g.NZAA);
  for (int i = 1; i <= g.NZAA; ++i)
    z[i - 1] = g.center + std::cos(pi * double(2 * i - 1) / double(2 * g.NZAA)) * 0.5 * g.gap;
  h->src_phys[2] = std::vector<double>(g.NZAA, -1.0);
  bool have = false;
  double hov = 0.0;
  for (auto& p : h->R.source_params)
    if (p.first == "HovEll") { have = true; hov = p.second; break; }
  if (!have && !h->R.source_params.empty()) return;
  std::vector<double> s1(g.NZAA);
  for (int i = 0; i < g.NZAA; ++i) s1[i] = hov * std::exp(-z[i] * hov) / (1.0 - std::exp(-hov)) - 1.0;
  h->src_phys[1] = s1;
}

// Constant K_hat terms of the mean systems (marching.f90:398-415): each source's
// Chebyshev coefficients (Compute_1dCheby_transform, marching.f90:845-866:
// REDFT10 / N, coefficient 0 halved; the first NZ), times dsca, through the
// truncated Cheb_IM(Iz, 0) rows of its equation.
void update_sources(coral_handle* h) {
  const Geometry& g = *h->G;
  const Recipe& R = h->R;
  h->src_missing.clear();
  std::vector<std::vector<double>> K(R.zero.size());
  for (const SourceTerm& t : R.sources) K[t.set].assign(h->zs[t.set].ops.T, 0.0);
  const long double pi = 3.141592653589793238462643383279502884L;
  for (const SourceTerm& t : R.sources) {
    auto it = h->src_phys.find(t.index);
    if (it == h->src_phys.end()) {
      char b[96];
      std::snprintf(b, sizeof(b), "source%02d is not defined (coral_set_source)", t.index);
      h->src_missing = b;
      continue;
    }
    const std::vector<double>& ph = it->second;
    const int N = g.NZAA;
    std::vector<double> c(g.NZ);
    for (int k = 0; k < g.NZ; ++k) {
      long double acc = 0.0L;
      for (int j = 0; j < N; ++j) acc += (long double)ph[j] * cosl(pi * ((long double)j + 0.5L) * k / N);
      c[k] = (double)(2.0L * acc) / N;
    }
    c[0] = c[0] * 0.5;
    const SystemOps& o = h->zs[t.set].ops;
    const Dense C = cheb_IM(g.NZ, g.center, g.gap, t.Iz, 0);
    const int oe = R.zero[t.set].orders[t.eqn];
    for (int rr = 0; rr < o.eq_size[t.eqn]; ++rr) {
      double acc = 0.0;
      for (int n = 0; n < g.NZ; ++n) acc += C[oe + rr][n] * (c[n] * t.dsca);
      K[t.set][o.eq_pos[t.eqn][rr]] += acc;
    }
  }
  // (the device vectors are made once, at creation, so captured graphs stay valid)
  for (size_t s = 0; s < R.zero.size(); ++s) {
    if (K[s].empty()) continue;
    if (!h->d_src[s]) h->d_src[s] = h->mem.get<double>(K[s].size());
    CK(cudaStreamSynchronize(h->stream));
    CK(cudaMemcpy(h->d_src[s], K[s].data(), K[s].size() * sizeof(double), cudaMemcpyHostToDevice));
    h->zs[s].dev.src = h->d_src[s];
  }
}

// every penalised variable's field from a mask on the device ([y][x][z])
void penal_fields(coral_handle* h, const double* mask) {
  const size_t n = (size_t)h->d.NYA * h->d.NXA * h->d.NZA;
  for (int f = 0; f < h->nF; ++f)
    if (h->penal_phys[f])
      launch_penal_field(n, mask, h->R.full[f].penal_strength, h->R.full[f].penal_width, h->penal_phys[f], h->stream);
  CK(cudaStreamSynchronize(h->stream));
}

// the z operations of surface values and vertical decompositions on Y2 rows
int launch_zfilters(coral_handle* h, int y0, int ny, cudaStream_t s) {
  const size_t vstride = (size_t)h->d.NYA * h->d.NXA * h->d.NZ;
  for (auto& z : h->zfilters) launch_zfilter(h->d, h->Y2 + z.var * vstride, z.extract, z.decomp, y0, ny, s);
  return (int)h->zfilters.size();
}

void setup(coral_handle* h, const std::string& eqs, const std::string& pars, const char* scheme, int device) {
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) throw CoralError(CORAL_ENODEV, "no CUDA device");
  if (device < 0 || device >= ndev) throw CoralError(CORAL_EBADARG, "device index out of range");
  h->device = device;
  CK(cudaSetDevice(device));
  CK(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
  h->P = parse_parameters(pars);
  h->R = parse_equations(eqs, h->smagorinsky);
  h->TB = ars_tableau(scheme && *scheme ? std::string(scheme) : h->P.scheme);
  if (h->TB.stages > kMaxStages) throw CoralError(CORAL_EUNSUPPORTED, "too many implicit stages");
  const Parameters& P = h->P;
  if (P.NX % 4 || P.NY % 4 || P.NZ % 4)
    throw CoralError(CORAL_EUNSUPPORTED, "NX, NY and NZ must be multiples of 4");
  h->G = std::make_unique<Geometry>(P);
  const Geometry& g = *h->G;
  if (!smooth23(g.NXAA) || !smooth23(g.NYAA) || !smooth23(g.NZAA))
    throw CoralError(CORAL_EUNSUPPORTED, "grid sizes must be of the form 2^a 3^b");
  h->d = Dims{g.NXH, g.NYAA, g.NXAA, g.NZ, g.NZAA};
  const Recipe& R = h->R;
  h->nF = (int)R.full.size();
  h->nQ = (int)R.quad.size();
  if (h->nF > kMaxFull || h->nQ > kMaxQuad || R.kxky.size() > (size_t)kMaxSets || R.zero.size() > (size_t)kMaxSets)
    throw CoralError(CORAL_EUNSUPPORTED, "recipe exceeds the built-in table sizes");
  DevAlloc& mem = h->mem;
  const size_t nsys = (size_t)g.NXH * g.NYAA;

  // geometry on the device
  h->d_kx = mem.upload(g.kx);
  h->d_ky = mem.upload(g.ky);
  h->d_wz = mem.upload(g.zweights());
  {
    std::vector<double> wi = g.zweights();
    for (double& w : wi) w = 1.0 / w;
    h->d_wzinv = mem.upload(wi);
  }
  std::vector<int> act_index(nsys, -1), act_list;
  for (int ix = 0; ix < g.NXH; ++ix)
    for (int iy = 0; iy < g.NYAA; ++iy)
      if (g.active(ix, iy)) {
        act_index[(size_t)ix * g.NYAA + iy] = (int)act_list.size();
        act_list.push_back(ix * g.NYAA + iy);
      }
  h->nact = (int)act_list.size();
  h->d_act_index = mem.upload(act_index);
  h->d_act_list = mem.upload(act_list);

  // transforms
  h->py = make_plan(mem, g.NYAA);
  h->px = make_plan(mem, g.NXAA);
  h->pz = make_plan(mem, g.NZAA);
  {
    std::vector<double2> t(g.NZAA);
    const long double pi = 3.141592653589793238462643383279502884L;
    for (int n = 0; n < g.NZAA; ++n) {
      long double a = -pi * (long double)n / (2.0L * (long double)g.NZAA);
      t[n] = make_double2((double)cosl(a), (double)sinl(a));
    }
    h->dct_tw = mem.upload(t);
  }

  // coupled kxky systems
  h->ks.resize(R.kxky.size());
  for (size_t s = 0; s < R.kxky.size(); ++s) {
    KSys& k = h->ks[s];
    k.ops = assemble_system(g, R, R.kxky[s]);
    k.T = k.ops.T;
    k.kl = k.ops.kl;
    k.ku = k.ops.ku;
    k.ldab = 2 * k.kl + k.ku + 1;
    k.ldab += k.ldab & 1;  // even column stride: every column starts on a 16-byte boundary
    if (k.kl > 63 || k.kl + k.ku > 127)
      throw CoralError(CORAL_EUNSUPPORTED, "band of the coupled system exceeds kl <= 63, kl+ku <= 127");
    k.M = upload_ell(mem, k.ops.M);
    k.L = upload_ell(mem, k.ops.L);
    k.NL = upload_ell(mem, k.ops.NLop);
    const size_t n = nsys * k.T;
    k.field = mem.get<double2>(n);
    k.aux = mem.get<double2>(n);
    CK(cudaMemset(k.field, 0, n * sizeof(double2)));
    CK(cudaMemset(k.aux, 0, n * sizeof(double2)));
    for (int i = 0; i < kMaxStages; ++i) {
      k.Kstd[i] = (i < h->TB.stages - 1) ? mem.get<double2>(n) : nullptr;
      k.Khat[i] = (i < h->TB.stages) ? mem.get<double2>(n) : nullptr;
    }
    k.real = k.ops.real_scalable && k.kl <= 16 && k.kl + k.ku <= 63 && std::getenv("CORAL_COMPLEX_FACTORS") == nullptr;
    k.ab = nullptr;
    k.abr = nullptr;
    k.rowflip = mem.upload(k.ops.row_flip);
    k.colflip = mem.upload(k.ops.col_flip);
    k.ncls = 1;
    k.Tc = k.T;
    k.kl_s = k.kl;
    k.ku_s = k.ku;
    k.ldab_s = k.ldab;
    k.wst = k.T;
    k.work = k.aux;
    k.Lp = k.L;
    k.colflip_cls = k.colflip;
    if (k.real && k.ops.ncls == 2 && k.ops.kl_cls <= 15 && k.ops.kl_cls + k.ops.ku_cls <= 31 &&
        std::getenv("CORAL_NO_CLASS_SPLIT") == nullptr) {
      k.ncls = 2;
      k.Tc = k.ops.Tc;
      k.kl_s = k.ops.kl_cls;
      k.ku_s = k.ops.ku_cls;
      k.ldab_s = 2 * k.kl_s + k.ku_s + 1;
      k.ldab_s += k.ldab_s & 1;
      k.wst = std::max(k.T, 2 * k.Tc);
      k.work = mem.get<double2>(nsys * k.wst);  // never aliases aux: k_kstd_out gathers from it into aux
      CK(cudaMemset(k.work, 0, nsys * k.wst * sizeof(double2)));
      k.row_pos = mem.upload(k.ops.row_cls_pos);
      k.col_pos = mem.upload(k.ops.col_cls_pos);
      k.cls_row = mem.upload(k.ops.cls_row);
      {
        std::vector<int> cc(2 * (size_t)k.Tc, -1);  // class position -> variable column
        for (int t = 0; t < k.T; ++t) cc[k.ops.col_cls_pos[t]] = t;
        k.cls_col = mem.upload(cc);
      }
      std::vector<unsigned char> cf(2 * (size_t)k.Tc, 0);
      for (int t = 0; t < k.T; ++t) cf[k.ops.col_cls_pos[t]] = k.ops.col_flip[t];
      k.colflip_cls = mem.upload(cf);
      EllOp lp = k.ops.L;
      for (int& c : lp.col)
        if (c >= 0) c = k.ops.col_cls_pos[c];
      k.Lp = upload_ell(mem, lp);
    }
    if (k.ncls == 2) {
      // K_std in tiles of kTileRows rows: per tile the window of solution columns
      // its rows of L touch, and L with columns relative to that window
      const int ntiles = (k.T + kTileRows - 1) / kTileRows;
      std::vector<int> tw(2 * (size_t)ntiles, 0);
      EllOp lw = k.ops.L;
      for (int tile = 0; tile < ntiles; ++tile) {
        const int t0 = tile * kTileRows, t1 = std::min(k.T, t0 + kTileRows);
        int lo = 1 << 30, hi = -1;
        for (int t = t0; t < t1; ++t)
          for (int kk = 0; kk < lw.width; ++kk) {
            const int c = lw.col[(size_t)t * lw.width + kk];
            if (c >= 0) { lo = std::min(lo, c); hi = std::max(hi, c); }
          }
        if (hi < 0) lo = 0;
        tw[2 * (size_t)tile] = lo;
        tw[2 * (size_t)tile + 1] = hi - lo + 1 > 0 ? hi - lo + 1 : 0;
        k.tile_lwin_max = std::max(k.tile_lwin_max, tw[2 * (size_t)tile + 1]);
        for (int t = t0; t < t1; ++t)
          for (int kk = 0; kk < lw.width; ++kk) {
            int& c = lw.col[(size_t)t * lw.width + kk];
            if (c >= 0) c -= lo;
          }
      }
      k.tile_win = mem.upload(tw);
      k.Lw = upload_gell(mem, lw);
      // the right-hand side in the same row tiles: the state window of M's
      // columns, the Chebyshev range and the quadratic variables of the NL
      // operator's columns (quad * NZ + n), and both operators relative to them
      std::vector<int> rw((size_t)ntiles * kRhsWin, 0);
      EllOp mw = k.ops.M, nw = k.ops.NLop;
      const int NZ = g.NZ;
      for (int tile = 0; tile < ntiles; ++tile) {
        const int t0 = tile * kTileRows, t1 = std::min(k.T, t0 + kTileRows);
        int mlo = 1 << 30, mhi = -1, nlo = 1 << 30, nhi = -1;
        std::vector<int> slot(kMaxQuad, -1), qs;
        for (int t = t0; t < t1; ++t) {
          for (int kk = 0; kk < mw.width; ++kk) {
            const int c = mw.col[(size_t)t * mw.width + kk];
            if (c >= 0) { mlo = std::min(mlo, c); mhi = std::max(mhi, c); }
          }
          for (int kk = 0; kk < nw.width; ++kk) {
            const int c = nw.col[(size_t)t * nw.width + kk];
            if (c < 0) continue;
            const int q = c / NZ, n = c - q * NZ;
            if (q >= kMaxQuad) throw CoralError(CORAL_EUNSUPPORTED, "too many quadratic variables");
            nlo = std::min(nlo, n);
            nhi = std::max(nhi, n);
            if (slot[q] < 0) { slot[q] = (int)qs.size(); qs.push_back(q); }
          }
        }
        if (mhi < 0) mlo = mhi = 0;
        if (nhi < 0) nlo = nhi = 0;
        const int mwid = mhi - mlo + 1, nwid = nhi - nlo + 1;
        int* r = rw.data() + (size_t)tile * kRhsWin;
        r[0] = mlo; r[1] = mwid; r[2] = nlo; r[3] = nwid; r[4] = (int)qs.size();
        for (size_t i = 0; i < qs.size(); ++i) r[5 + i] = qs[i];
        k.rhs_win_max = std::max(k.rhs_win_max, mwid + (int)qs.size() * nwid);
        for (int t = t0; t < t1; ++t) {
          for (int kk = 0; kk < mw.width; ++kk) {
            int& c = mw.col[(size_t)t * mw.width + kk];
            if (c >= 0) c -= mlo;
          }
          for (int kk = 0; kk < nw.width; ++kk) {
            int& c = nw.col[(size_t)t * nw.width + kk];
            if (c < 0) continue;
            const int q = c / NZ, n = c - q * NZ;
            c = slot[q] * nwid + n - nlo;
          }
        }
      }
      k.rhs_win = mem.upload(rw);
      k.Mw = upload_ell(mem, mw);
      k.NLw = upload_ell(mem, nw);
      k.NLg = upload_gell(mem, nw);
    }
    if (k.ncls == 2) {
      // thread-per-block layouts: groups of 32 blocks (block = 2 act + class) side by side
      const size_t ngroups = ((size_t)h->nact * 2 + 31) / 32;
      k.abr = mem.get<double>(ngroups * k.Tc * k.ldab_s * 32);
      k.dpiv = mem.get<unsigned char>(ngroups * k.Tc * 32);
      k.work2 = mem.get<double2>(ngroups * k.Tc * 32);
      k.cmask = mem.get<unsigned long long>(k.Tc);
      k.lmask = mem.get<unsigned>(k.Tc);
      k.umask = mem.get<unsigned>(k.Tc);
      CK(cudaMemset(k.work2, 0, ngroups * k.Tc * 32 * sizeof(double2)));
    } else {
      if (k.real) k.abr = mem.get<double>((size_t)h->nact * k.Tc * k.ldab_s);
      else k.ab = mem.get<double2>((size_t)h->nact * k.T * k.ldab);
      // pivot rows padded to 8 bytes, one row per system
      k.dpiv = mem.get<unsigned char>((size_t)h->nact * ((k.Tc + 7) & ~7));
    }
    k.info = mem.get<int>((size_t)std::max(h->nact, 1));
    for (int v = 0; v < k.ops.nV; ++v) {
      std::vector<int> tt;
      std::vector<double> tv;
      stencil_tab(k.ops, v, g.NZ, tt, tv);
      k.tab_t.push_back(tt);
      k.tab_v.push_back(tv);
      k.d_tab_t.push_back(mem.upload(tt));
      k.d_tab_v.push_back(mem.upload(tv));
      k.d_var_pos.push_back(mem.upload(k.ops.var_pos[v]));
      // square stencil rows (lower triangular)
      int nc = k.ops.var_size[v];
      std::vector<int> sc((size_t)nc * kTabW, -1);
      std::vector<double> sv((size_t)nc * kTabW, 0.0);
      for (int r = 0; r < nc; ++r) {
        int q = 0;
        for (auto& e : k.ops.stencil_rows[v][r])
          if (e.first < nc) { sc[(size_t)r * kTabW + q] = e.first; sv[(size_t)r * kTabW + q] = e.second; ++q; }
      }
      k.d_sq_col.push_back(mem.upload(sc));
      k.d_sq_val.push_back(mem.upload(sv));
    }
  }
  // mean systems
  h->zs.resize(R.zero.size());
  for (size_t s = 0; s < R.zero.size(); ++s) {
    ZSys& z = h->zs[s];
    z.ops = assemble_system(g, R, R.zero[s]);
    for (auto& gp : z.ops.M.groups)
      if (gp.first || gp.second) throw CoralError(CORAL_EPARSE, "x/y-derivative in a mean-field recipe");
    for (auto& gp : z.ops.L.groups)
      if (gp.first || gp.second) throw CoralError(CORAL_EPARSE, "x/y-derivative in a mean-field recipe");
    ZeroSysDev& dz = z.dev;
    dz.T = z.ops.T;
    dz.kl = z.ops.kl;
    dz.ku = z.ops.ku;
    dz.ldab = 2 * dz.kl + dz.ku + 1;
    dz.M = upload_ell(mem, z.ops.M);
    dz.L = upload_ell(mem, z.ops.L);
    dz.NL = upload_ell(mem, z.ops.NLop);
    dz.field = mem.get<double>(dz.T);
    dz.aux = mem.get<double>(dz.T);
    CK(cudaMemset(dz.field, 0, dz.T * sizeof(double)));
    CK(cudaMemset(dz.aux, 0, dz.T * sizeof(double)));
    for (int i = 0; i < kMaxStages; ++i) {
      dz.Kstd[i] = (i < h->TB.stages - 1) ? mem.get<double>(dz.T) : nullptr;
      dz.Khat[i] = (i < h->TB.stages) ? mem.get<double>(dz.T) : nullptr;
    }
    dz.ab = mem.get<double>((size_t)dz.T * dz.ldab);
    dz.dpiv = mem.get<unsigned char>(dz.T);
    dz.src = nullptr;
    for (int v = 0; v < z.ops.nV; ++v) {
      std::vector<int> tt;
      std::vector<double> tv;
      stencil_tab(z.ops, v, g.NZ, tt, tv);
      z.tab_t.push_back(tt);
      z.tab_v.push_back(tv);
      z.d_tab_t.push_back(mem.upload(tt));
      z.d_tab_v.push_back(mem.upload(tv));
    }
  }
  h->zinfo = mem.get<int>(kMaxSets);

  // full variables
  std::vector<FullVarDev> fv(h->nF);
  for (int f = 0; f < h->nF; ++f) {
    const FullVar& F = R.full[f];
    if (F.terms.size() > (size_t)kMaxFullTerms) throw CoralError(CORAL_EUNSUPPORTED, "too many terms in a full variable");
    fv[f].nterms = (int)F.terms.size();
    for (size_t t = 0; t < F.terms.size(); ++t) {
      const FullTerm& ft = F.terms[t];
      if (ft.mz != 0)  // compute_full_variables_in_physical_space applies no mz (marching.f90:436-503)
        throw CoralError(CORAL_EUNSUPPORTED, "mz in a full-variable build is not supported");
      FullTermDev& o = fv[f].term[t];
      o.zero_kind = ft.zero_kind ? 1 : 0;
      o.dx = ft.dx;
      o.dy = ft.dy;
      o.dsca = ft.dsca;
      if (ft.zero_kind) {
        auto loc = R.zero_loc.at(R.zero_vars[ft.var]);
        o.set = loc.first;
        o.tab_t = h->zs[loc.first].d_tab_t[loc.second];
        o.tab_v = h->zs[loc.first].d_tab_v[loc.second];
        if (ft.dz != 0) {  // built by k_zero_dz, read back through an identity stencil
          if (h->zs.size() + h->zdz_jobs.size() >= (size_t)kMaxSets)
            throw CoralError(CORAL_EUNSUPPORTED, "too many z-derivative terms in the full-variable builds");
          if (!h->d_tab_id_t) {
            std::vector<int> tt((size_t)g.NZ * kTabW, -1);
            std::vector<double> tv((size_t)g.NZ * kTabW, 0.0);
            for (int n = 0; n < g.NZ; ++n) {
              tt[(size_t)n * kTabW] = n;
              tv[(size_t)n * kTabW] = 1.0;
            }
            h->d_tab_id_t = mem.upload(tt);
            h->d_tab_id_v = mem.upload(tv);
          }
          // (the reference scales a mean term by dsca after its derivatives: the
          // build applies o.dsca to the differentiated profile)
          coral_handle::ZDzJob j{o.set, ft.dz, o.tab_t, o.tab_v, 1.0, mem.get<double>(g.NZ)};
          o.set = (int)(h->zs.size() + h->zdz_jobs.size());
          o.tab_t = h->d_tab_id_t;
          o.tab_v = h->d_tab_id_v;
          h->zdz_jobs.push_back(j);
        }
      } else {
        auto it = R.kxky_loc.find(R.kxky_vars[ft.var]);
        if (it == R.kxky_loc.end()) throw CoralError(CORAL_EPARSE, "kxky variable in no coupled system");
        o.set = it->second.first;
        o.tab_t = h->ks[it->second.first].d_tab_t[it->second.second];
        o.tab_v = h->ks[it->second.first].d_tab_v[it->second.second];
        if (ft.dz != 0) {
          // built by k_full_dz (dsca applied before the derivatives, as the
          // reference does), read back through an identity stencil
          if (h->ks.size() + h->dz_jobs.size() >= (size_t)kMaxSets)
            throw CoralError(CORAL_EUNSUPPORTED, "too many z-derivative terms in the full-variable builds");
          if (!h->d_tab_id_t) {
            std::vector<int> tt((size_t)g.NZ * kTabW, -1);
            std::vector<double> tv((size_t)g.NZ * kTabW, 0.0);
            for (int n = 0; n < g.NZ; ++n) {
              tt[(size_t)n * kTabW] = n;
              tv[(size_t)n * kTabW] = 1.0;
            }
            h->d_tab_id_t = mem.upload(tt);
            h->d_tab_id_v = mem.upload(tv);
          }
          coral_handle::DzJob j{o.set, h->ks[o.set].T, ft.dz, o.tab_t, o.tab_v, o.dsca,
                                mem.get<double2>((size_t)g.NXH * g.NYAA * g.NZ)};
          o.set = (int)(h->ks.size() + h->dz_jobs.size());
          o.tab_t = h->d_tab_id_t;
          o.tab_v = h->d_tab_id_v;
          o.dsca = 1.0;
          h->dz_jobs.push_back(j);
        }
      }
    }
  }
  h->d_fv = mem.upload(fv);
  h->fv_single = h->nF > 0;
  for (int f = 0; f < h->nF; ++f) {
    int nk = 0;
    for (int t = 0; t < fv[f].nterms; ++t) nk += fv[f].term[t].zero_kind ? 0 : 1;
    if (nk != 1 || fv[f].term[fv[f].nterms - 1].zero_kind) h->fv_single = false;
  }
  // quadratic variables
  h->quads.nq = h->nQ;
  h->quads.ke_q[0] = h->quads.ke_q[1] = h->quads.ke_q[2] = -1;
  for (int q = 0; q < h->nQ; ++q) {
    h->quads.v1[q] = R.quad[q].v1;
    h->quads.v2[q] = R.quad[q].v2;
    if (R.quad[q].remove_mean) h->zmean_quads.push_back(q);
    if (R.quad[q].name == "uu") h->quads.ke_q[0] = q;
    if (R.quad[q].name == "vv") h->quads.ke_q[1] = q;
    if (R.quad[q].name == "ww") h->quads.ke_q[2] = q;
  }
  // full variables that are not plain transforms
  {
    std::vector<double> zg(g.NZAA);
    const double pi = 4.0 * std::atan(1.0);
    for (int i = 1; i <= g.NZAA; ++i)
      zg[i - 1] = g.center + std::cos(pi * double(2 * i - 1) / double(2 * g.NZAA)) * 0.5 * g.gap;
    h->d_zgrid = mem.upload(zg);
    h->penal_phys.assign(h->nF, nullptr);
    h->quads.st_n = 0;
    for (int f = 0; f < h->nF; ++f) {
      const FullVar& F = R.full[f];
      if (F.penal || F.smago) {
        if (h->quads.st_n >= kMaxStatic) throw CoralError(CORAL_EUNSUPPORTED, "too many penalised variables");
        const int k = h->quads.st_n++;
        h->quads.st_var[k] = f;
        h->quads.st_prof[k] = F.smago ? 1 : 0;
        if (F.smago) {
          h->smago_var = f;
          h->smago_prof = mem.get<double>(g.NZAA);
          CK(cudaMemset(h->smago_prof, 0, g.NZAA * sizeof(double)));
          h->smago_part = mem.get<double>((size_t)g.NYAA * g.NZAA);
          h->quads.st_src[k] = h->smago_prof;
          for (int j = 0; j < h->nF; ++j) {
            const std::string& n = R.full[j].name;
            if (n == "dxUfull" || n == "dyUfull" || n == "dxVfull" || n == "dyVfull") h->smago_src.push_back(j);
          }
        } else {
          h->penal_phys[f] = mem.get<double>((size_t)g.NYAA * g.NXAA * g.NZAA);
          h->quads.st_src[k] = h->penal_phys[f];
        }
      } else if (F.extract || F.decomp) {
        h->zfilters.push_back({f, F.extract, F.decomp});
      }
    }
  }
  // sources of the mean equations: the reference's default definitions, then the
  // constant K_hat terms
  h->d_src.assign(R.zero.size(), nullptr);
  default_sources(h);
  update_sources(h);
  // transform buffers
  const int nmax = std::max(std::max(h->nF, h->nQ), 1);
  h->Y1 = mem.get<double2>((size_t)nmax * g.NYAA * g.NXH * g.NZ);
  h->Y2 = mem.get<double>((size_t)nmax * g.NYAA * g.NXAA * g.NZ);
  h->fphys = mem.get<double>((size_t)std::max(h->nF, 1) * g.NYAA * g.NXAA * g.NZAA);
  h->qspec = mem.get<double2>((size_t)std::max(h->nQ, 1) * nsys * g.NZ);
  h->tmp_spec = mem.get<double2>(nsys * g.NZ);
  h->tmp_phys = mem.get<double>((size_t)g.NYAA * g.NXAA * g.NZAA);
  h->n_ke_partial = (size_t)((g.NXAA + 1) / 2) * g.NYAA * 3;
  h->ke_partial = mem.get<double>(h->n_ke_partial);
  h->ke_total = mem.get<double>(1);
  CK(cudaMemset(h->ke_partial, 0, h->n_ke_partial * sizeof(double)));
  // |u|, |v|, |w| / wz and the Smagorinsky viscosity
  h->cfl_bits = mem.get<unsigned long long>(4);
  CK(cudaMemset(h->cfl_bits, 0, 4 * sizeof(unsigned long long)));
  h->flags = mem.get<unsigned int>(1);
  CK(cudaMemset(h->flags, 0, sizeof(unsigned int)));
  h->ts_ncta = z_fused_ctas(h->d);
  h->ts_partial = mem.get<double>(h->ts_ncta * kMaxTs);
  h->ts_out = mem.get<double>(kMaxTs);
  CK(cudaMemset(h->ts_out, 0, kMaxTs * sizeof(double)));
  CK(cudaMallocHost(&h->h_pin, (kMaxTs + 5) * sizeof(double)));
  // penalisation fields from the reference's default mask (coral_set_penalisation_mask
  // replaces it)
  if (std::any_of(R.full.begin(), R.full.end(), [](const FullVar& F) { return F.penal; })) {
    launch_penal_default(h->d, g.Lx, g.Ly, h->d_zgrid, h->tmp_phys, h->stream);
    penal_fields(h, h->tmp_phys);
  }
  // timings%init (timeKeeping.f90:57-70): dt_current = dt = dt_max, t = 0, step 1
  h->dt_current = h->dt_target = P.dt_max;
  h->time = 0.0;
  h->i_timestep = 1;
  CK(cudaDeviceSynchronize());
}

StateSet state_set(coral_handle* h, bool use_field) {
  StateSet st{};
  for (size_t s = 0; s < h->ks.size(); ++s) {
    st.k[s] = use_field ? h->ks[s].field : h->ks[s].aux;
    st.kT[s] = h->ks[s].T;
  }
  for (size_t j = 0; j < h->dz_jobs.size(); ++j) {  // the dz terms' buffers (pseudo-systems)
    st.k[h->ks.size() + j] = h->dz_jobs[j].out;
    st.kT[h->ks.size() + j] = h->d.NZ;
  }
  for (size_t s = 0; s < h->zs.size(); ++s) st.z[s] = use_field ? h->zs[s].dev.field : h->zs[s].dev.aux;
  for (size_t j = 0; j < h->zdz_jobs.size(); ++j) st.z[h->zs.size() + j] = h->zdz_jobs[j].out;
  return st;
}

// the dz terms of the full-variable builds from the state set st (before the build)
int launch_dz_jobs(coral_handle* h, const StateSet& st) {
  for (auto& j : h->dz_jobs)
    launch_full_dz(h->d, st.k[j.set], j.T, j.tab_t, j.tab_v, j.dsca, j.order, h->G->gap, j.out, h->stream);
  for (auto& j : h->zdz_jobs)
    launch_zero_dz(h->d.NZ, st.z[j.set], j.tab_t, j.tab_v, j.dsca, j.order, h->G->gap, j.out, h->stream);
  return (int)(h->dz_jobs.size() + h->zdz_jobs.size());
}

// inverse transforms of all full variables built from field (stage 0) or aux
int full_vars_to_phys(coral_handle* h, bool use_field, bool cfl) {
  const Dims& d = h->d;
  const StateSet st = state_set(h, use_field);
  const int ndz = launch_dz_jobs(h, st);
  launch_inv_y(d, h->nF, h->d_fv, st, nullptr, h->d_kx, h->d_ky, h->Y1, h->py, h->stream,
               h->fv_single && !h->tune.inv_y_loop);
  launch_inv_x(d, h->nF, h->Y1, h->Y2, h->px, h->stream);
  const int nzf = launch_zfilters(h, 0, d.NYA, h->stream);
  if (cfl) CK(cudaMemsetAsync(h->cfl_bits, 0, 4 * sizeof(unsigned long long), h->stream));
  launch_inv_z(d, h->nF, h->Y2, h->fphys, h->pz, h->dct_tw, h->d_wz, cfl ? h->cfl_bits : nullptr, h->stream);
  launch_static_phys(d, h->quads, h->fphys, h->stream);
  return 3 + ndz + nzf + (h->quads.st_n > 0 ? 1 : 0);
}

constexpr int kProfileClasses = 11;  // coral_profile_step

struct PhaseTimer {
  cudaStream_t s;
  std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> ev;
  void begin(int k) {
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaEventRecord(a, s);
    ev.push_back({k, {a, b}});
  }
  void end() { cudaEventRecord(ev.back().second.second, s); }
};

// Arguments of the stage-i kernels of coupled kxky system k.
NLArgs make_nl_args(coral_handle* h, KSys& k, int i) {
  NLArgs na{};
  na.d = h->d;
  na.T = k.T;
  na.NL = k.NL;
  na.qspec = h->qspec;
  na.kx = h->d_kx;
  na.ky = h->d_ky;
  na.act_index = h->d_act_index;
  na.Khat = k.Khat[i];
  na.nq = h->nQ;
  return na;
}

SolveArgs make_solve_args(coral_handle* h, KSys& k, int i, double dt) {
  const int S = h->TB.stages;
  const bool last = (i == S - 1);
  SolveArgs sa{};
  sa.d = h->d;
  sa.T = k.T;
  sa.kl = k.real ? k.kl_s : k.kl;
  sa.ku = k.real ? k.ku_s : k.ku;
  sa.ldab = k.real ? k.ldab_s : k.ldab;
  sa.M = k.M;
  sa.L = k.L;
  sa.field = k.field;
  sa.out = last ? k.field : k.aux;
  sa.work = k.work;
  sa.Kstd_out = last ? nullptr : k.Kstd[i];
  sa.nprev = i;
  for (int j = 0; j <= i; ++j) {
    sa.Kstd[j] = k.Kstd[j];
    sa.Khat[j] = k.Khat[j];
    sa.ca[j] = (j < i) ? dt * h->TB.a(i, j) : 0.0;
    sa.ch[j] = dt * h->TB.ahat(i + 1, j);
  }
  sa.ab = k.ab;
  sa.dpiv = k.dpiv;
  sa.act_index = h->d_act_index;
  sa.act_list = h->d_act_list;
  sa.nact = h->nact;
  sa.last_stage = last ? 1 : 0;
  sa.kx = h->d_kx;
  sa.ky = h->d_ky;
  sa.flags = h->flags;
  sa.abr = k.abr;
  sa.rowflip = k.rowflip;
  sa.colflip = k.colflip;
  sa.ncls = k.ncls;
  sa.Tc = k.Tc;
  sa.wst = k.wst;
  sa.row_pos = k.row_pos;
  sa.col_pos = k.col_pos;
  sa.colflip_cls = k.colflip_cls;
  sa.Lp = k.Lp;
  sa.work2 = k.work2;
  sa.nblk = k.ncls * h->nact;
  sa.cls_col = k.cls_col;
  sa.lmask = k.lmask;
  sa.umask = k.umask;
  sa.tile_win = k.tile_win;
  sa.tile_lwin_max = k.tile_lwin_max;
  sa.rhs_win = k.rhs_win;
  sa.rhs_win_max = k.rhs_win_max;
  sa.Mw = k.Mw;
  sa.NLw = k.NLw;
  sa.NLg = k.NLg;
  // CORAL_GENERIC_TILES=1: the run-time forms of the tile kernels (tests cover
  // them with the plane-layer recipes, whose layouts are otherwise compiled)
  sa.generic_tiles = std::getenv("CORAL_GENERIC_TILES") != nullptr || h->tune.generic_tiles;
  sa.subst_rt = h->tune.subst_rt;
  sa.Lw = k.Lw;
  {
    const int kv = sa.kl + sa.ku;
    const int u_rows = (kv + 2) & ~1, l_rows = ((kv + 1 + sa.kl + 1) & ~1) - ((kv + 1) & ~1);
    sa.ring_cols = k.ncls * std::max(u_rows, l_rows);
  }
  return sa;
}

// Stage i of one_step_beyond (marching.f90:9-28) in three phases, so that an
// ensemble can run the band substitutions of all its members as one launch:
//   pre   full variables -> physical space, products, forward transforms
//         (compute_NL_terms_to_K_hat), and the right-hand side with the NL
//         assembly (or, for complex factors, NL assembly + the whole solve);
//   subst the band substitutions (backsolve_to_aux);
//   post  K_std = L aux and the stage output (stif_aux_to_K_std), the mean systems.
int enqueue_stage_pre(coral_handle* h, int i, double dt, PhaseTimer* pt) {
  auto B = [&](int k) { if (pt) pt->begin(k); };
  auto E = [&]() { if (pt) pt->end(); };
  const Dims& d = h->d;
  const Geometry& g = *h->G;
  int nl = 0;
  const int S = h->TB.stages;
  const double scale = 1.0 / ((double)g.NXAA * (double)g.NYAA * (double)g.NZAA);
  const bool last = (i == S - 1);
  // the y-chunked pipeline (eager phase timing keeps whole passes, one kernel per phase)
  const bool chunked = !pt && h->tune.y_chunks > 1 && h->yfork && !h->closure && h->zform == 0 && h->smago_var < 0 &&
                       h->tune.inv_x_tiles == 1 && (size_t)d.NXA * d.NYA >= (size_t)288 * 288;
  if (chunked) {
    StateSet st = state_set(h, i == 0);
    nl += launch_dz_jobs(h, st);
    launch_inv_y(d, h->nF, h->d_fv, st, nullptr, h->d_kx, h->d_ky, h->Y1, h->py, h->stream, h->fv_single && !h->tune.inv_y_loop);
    if (last) CK(cudaMemsetAsync(h->cfl_bits, 0, 4 * sizeof(unsigned long long), h->stream));
    QuadDesc q = h->quads;
    q.ts_partial = (i == 0 && q.ts_n > 0) ? h->ts_partial : nullptr;
    // a band of y rows needs only its own rows through the three passes: Y1 rows
    // -> Y2 rows (x c2r), Y2 rows in place (z), Y2 rows -> Y1 rows (x r2c)
    const int nch = std::min(h->tune.y_chunks, d.NYA);
    CK(cudaEventRecord(h->yfork, h->stream));
    for (int k = 0; k < kYStreams; ++k) CK(cudaStreamWaitEvent(h->ystream[k], h->yfork, 0));
    for (int c = 0; c < nch; ++c) {
      const int y0 = (int)((long long)d.NYA * c / nch), y1 = (int)((long long)d.NYA * (c + 1) / nch);
      cudaStream_t ss = h->ystream[c % kYStreams];
      launch_inv_x_rows(d, h->nF, h->Y1, h->Y2, h->px, h->tune.x_plan, y0, y1 - y0, ss);
      nl += launch_zfilters(h, y0, y1 - y0, ss);
      launch_z_fused(d, h->nF, q, h->Y2, h->Y2, h->pz, h->dct_tw, h->d_wz, h->d_wzinv, last ? h->cfl_bits : nullptr,
                     i == 0 ? h->ke_partial : nullptr, ss, h->tune.z_batch6, y0, y1 - y0);
      launch_fwd_x(d, h->nQ, h->Y2, h->Y1, h->px, ss, h->tune.x_plan, y0, y1 - y0);
    }
    for (int k = 0; k < kYStreams; ++k) {
      CK(cudaEventRecord(h->yjoin[k], h->ystream[k]));
      CK(cudaStreamWaitEvent(h->stream, h->yjoin[k], 0));
    }
    launch_fwd_y(d, h->nQ, h->Y1, h->qspec, scale, h->py, h->stream, h->tune.fwd_y_grid);
    nl += 2 + 3 * nch;
  }
  if (!chunked) {
    {
      StateSet st = state_set(h, i == 0);
      B(0); nl += launch_dz_jobs(h, st);
      launch_inv_y(d, h->nF, h->d_fv, st, nullptr, h->d_kx, h->d_ky, h->Y1, h->py, h->stream, h->fv_single && !h->tune.inv_y_loop); E();
      B(1); launch_inv_x(d, h->nF, h->Y1, h->Y2, h->px, h->stream, h->tune.x_plan, h->tune.inv_x_tiles);
      nl += launch_zfilters(h, 0, d.NYA, h->stream); E();
      // the CFL maxima reported after a step are those of its last stage's fields
      // (each stage's evaluation replaces them): only the last stage computes them
      if (last) CK(cudaMemsetAsync(h->cfl_bits, 0, 4 * sizeof(unsigned long long), h->stream));
      nl += 2;
    }
    // the Smagorinsky viscosity needs every column's physical fields first: the
    // inverse z transforms to HBM, the profile, then the z passes with the
    // profile in nuSmago's place (marching.f90:516-541)
    const bool smago_now = h->smago_var >= 0 && !h->closure;
    if (smago_now) {
      B(3);
      // only the variables the viscosity is formed from
      const size_t ystride = (size_t)d.NYA * d.NXA * d.NZ, pstride = (size_t)d.NYA * d.NXA * d.NZA;
      for (int v : h->smago_src)
        launch_inv_z(d, 1, h->Y2 + v * ystride, h->fphys + v * pstride, h->pz, h->dct_tw, h->d_wz, nullptr, h->stream);
      launch_smago(d, h->fphys, h->smago_src.data(), (int)h->smago_src.size(), h->smago_prefactor, h->smago_part,
                   h->smago_prof, last ? h->cfl_bits + 3 : nullptr, h->stream);
      E();
      nl += 2 + (int)h->smago_src.size();
    }
    // z passes fused (inverse DCT, CFL maxima, products, KE, forward DCT); the
    // quadratic variables overwrite Y2 in place, each CTA reading and writing only
    // its own (y, x pair) columns
    B(3);
    if (h->closure) {
      // unfused z passes around the network: physical fields to HBM, the
      // network's subgrid parts, then the products (plus those parts) forward
      launch_inv_z(d, h->nF, h->Y2, h->fphys, h->pz, h->dct_tw, h->d_wz, last ? h->cfl_bits : nullptr, h->stream);
      if (h->smago_var >= 0) {
        launch_smago(d, h->fphys, h->smago_src.data(), (int)h->smago_src.size(), h->smago_prefactor, h->smago_part,
                     h->smago_prof, last ? h->cfl_bits + 3 : nullptr, h->stream);
        nl += 2;
      }
      if (h->quads.st_n > 0) {
        launch_static_phys(d, h->quads, h->fphys, h->stream);
        ++nl;
      }
      closure_infer(closure_impl(h->closure), h->fphys, d.NYA, d.NXA, d.NZA, h->tau, h->stream);
      QuadDesc q = h->quads;
      q.ts_partial = nullptr;
      q.tau = h->tau;
      launch_fwd_z(d, h->nF, q, h->fphys, h->Y2, h->pz, h->dct_tw, h->d_wz, i == 0 ? h->ke_partial : nullptr,
                   h->stream);
      nl += 2;
    } else if (h->zform == 1) {
      // the tensor-core form: inverse contraction into the physical fields,
      // then products and the forward contraction back into Y2
      QuadDesc q = h->quads;
      q.ts_partial = nullptr;
      const bool ts = (i == 0 && q.ts_n > 0);
      launch_zsplit_inv(d, h->nF, q, h->Y2, h->fphys, h->zmat_inv, h->d_wz, h->d_wzinv,
                        last ? h->cfl_bits : nullptr, ts ? h->ts_partial_split : nullptr, h->flags, h->stream);
      launch_zsplit_fwd(d, h->nF, q, h->fphys, h->Y2, h->zmat_fwd, h->d_wz,
                        i == 0 ? h->ke_partial_split : nullptr, ts ? h->ts_partial_split : nullptr,
                        (long long)h->ts_inv_rows, h->flags, h->stream);
      ++nl;
    } else {
      // the first stage's fields also give the timeseries objects
      QuadDesc q = h->quads;
      q.ts_partial = (i == 0 && q.ts_n > 0) ? h->ts_partial : nullptr;
      launch_z_fused(d, h->nF, q, h->Y2, h->Y2, h->pz, h->dct_tw, h->d_wz, h->d_wzinv,
                     last ? h->cfl_bits : nullptr, i == 0 ? h->ke_partial : nullptr, h->stream, h->tune.z_batch6);
    }
    E();
    B(4); launch_fwd_x(d, h->nQ, h->Y2, h->Y1, h->px, h->stream, h->tune.x_plan); E();
    B(5); launch_fwd_y(d, h->nQ, h->Y1, h->qspec, scale, h->py, h->stream, h->tune.fwd_y_grid); E();
    nl += 3;
  }
  for (int q : h->zmean_quads) {
    launch_remove_zmean(d, h->qspec + (size_t)q * d.NXH * d.NYA * d.NZ, h->stream);
    ++nl;
  }
  for (auto& k : h->ks) {
    NLArgs na = make_nl_args(h, k, i);
    SolveArgs sa = make_solve_args(h, k, i, dt);
    if (k.real) {
      B(7); launch_rhs_nl(sa, na, h->stream); E();
      ++nl;
    } else {
      B(6); launch_nl(na, h->stream); E();
      B(7); launch_solve(sa, h->stream); E();
      nl += 2;
    }
  }
  return nl;
}

int enqueue_stage_subst(coral_handle* h, int i, double dt, PhaseTimer* pt) {
  int nl = 0;
  for (auto& k : h->ks)
    if (k.real) {
      SolveArgs sa = make_solve_args(h, k, i, dt);
      if (pt) pt->begin(9);
      launch_subst(sa, h->stream);
      if (pt) pt->end();
      ++nl;
    }
  return nl;
}

int enqueue_stage_post(coral_handle* h, int i, double dt, PhaseTimer* pt) {
  int nl = 0;
  const int S = h->TB.stages;
  const bool last = (i == S - 1);
  for (auto& k : h->ks)
    if (k.real) {
      SolveArgs sa = make_solve_args(h, k, i, dt);
      if (pt) pt->begin(10);
      launch_kstd_out(sa, h->stream);
      if (pt) pt->end();
      ++nl;
    }
  if (!h->zs.empty()) {
    ZeroArgs za{};
    za.nsys = (int)h->zs.size();
    for (size_t s = 0; s < h->zs.size(); ++s) za.sys[s] = h->zs[s].dev;
    za.qspec = h->qspec;
    za.d = h->d;
    za.stage = i;
    for (int j = 0; j <= i; ++j) {
      za.ca[j] = (j < i) ? dt * h->TB.a(i, j) : 0.0;
      za.ch[j] = dt * h->TB.ahat(i + 1, j);
    }
    za.last_stage = last ? 1 : 0;
    if (pt) pt->begin(8);
    launch_zero_step(za, h->stream);
    if (pt) pt->end();
    ++nl;
  }
  return nl;
}

// after the stages: the kx = 0 projection (when enabled) and the timeseries
// totals of the step
int enqueue_step_end(coral_handle* h) {
  const Geometry& g = *h->G;
  int nl = 0;
  if (h->hermitian_kx0)
    for (auto& k : h->ks) {
      launch_hermitian_kx0(k.field, h->d.NYA, k.T, h->stream);
      ++nl;
    }
  if (h->quads.ts_n > 0) {
    if (h->zform == 1)
      launch_ts_reduce(h->ts_partial_split, h->ts_rows_split, h->quads.ts_n, 1.0 / ((double)g.NXAA * (double)g.NYAA),
                       h->ts_out, h->stream);
    else
      launch_ts_reduce(h->ts_partial, h->ts_ncta, h->quads.ts_n, 1.0 / ((double)g.NXAA * (double)g.NYAA), h->ts_out,
                       h->stream);
    ++nl;
  }
  h->zform_last = h->zform;
  CK(cudaGetLastError());
  return nl;
}

int enqueue_step(coral_handle* h, double dt, PhaseTimer* pt = nullptr) {
  int nl = 0;
  for (int i = 0; i < h->TB.stages; ++i) {
    nl += enqueue_stage_pre(h, i, dt, pt);
    nl += enqueue_stage_subst(h, i, dt, pt);
    nl += enqueue_stage_post(h, i, dt, pt);
  }
  return nl + enqueue_step_end(h);
}

// Select the z-transform form; the tensor-core form needs NZ and NZAA to be
// multiples of 96 (its output tiles) and allocates its digit tables and
// partial-sum arrays on first use.
void set_z_transform(coral_handle* h, int form) {
  if (form != 0 && form != 1) throw CoralError(CORAL_EBADARG, "z transform form must be 0 (FP64) or 1 (int8 digits)");
  const Geometry& g = *h->G;
  if (form == 1) {
    if (h->quads.st_n > 0)
      throw CoralError(CORAL_EUNSUPPORTED, "the tensor-core z transform does not take penalised or Smagorinsky variables");
    if (!zsplit_supported(g.NZ, g.NZAA))
      throw CoralError(CORAL_EUNSUPPORTED, "the tensor-core z transform needs NZ and 3 NZ / 2 to be multiples of 96");
    if (!h->zmat_inv) {
      h->zmat_inv = h->mem.upload(zsplit_matrix_digits(g.NZ, g.NZAA, false, g.NZAA));
      h->zmat_fwd = h->mem.upload(zsplit_matrix_digits(g.NZAA, g.NZ, true, g.NZAA));
      const long long ncol = (long long)g.NYAA * g.NXAA;
      const size_t nfwd = zsplit_ctas(ncol, h->nQ);
      h->ts_inv_rows = zsplit_ctas(ncol, h->nF);
      h->ts_rows_split = h->ts_inv_rows + nfwd;
      h->n_ke_split = nfwd * 3;
      h->ke_partial_split = h->mem.get<double>(h->n_ke_split);
      h->ts_partial_split = h->mem.get<double>(h->ts_rows_split * kMaxTs);
      CK(cudaMemset(h->ke_partial_split, 0, h->n_ke_split * sizeof(double)));
      CK(cudaMemset(h->ts_partial_split, 0, h->ts_rows_split * kMaxTs * sizeof(double)));
    }
  }
  h->zform = form;
  if (h->graph) {
    cudaGraphExecDestroy(h->graph);
    h->graph = nullptr;
  }
}

void factorize(coral_handle* h, double dt) {
  const Dims& d = h->d;
  const double zsca = -dt * h->TB.a(0, 0);
  for (auto& k : h->ks) {
    FactorArgs fa{};
    fa.d = d;
    fa.T = k.T;
    fa.kl = k.real ? k.kl_s : k.kl;
    fa.ku = k.real ? k.ku_s : k.ku;
    fa.ldab = k.real ? k.ldab_s : k.ldab;
    fa.ncls = k.ncls;
    fa.Tc = k.Tc;
    fa.cls_row = k.cls_row;
    fa.col_pos = k.col_pos;
    fa.tpb = k.work2 != nullptr;
    fa.window = h->tune.factor_window;
    fa.cmask = k.cmask;
    fa.lmask = k.lmask;
    fa.umask = k.umask;
    fa.nact = h->nact;
    fa.M = k.M;
    fa.L = k.L;
    fa.zsca = zsca;
    fa.act_list = h->d_act_list;
    fa.ab = k.ab;
    fa.dpiv = k.dpiv;
    fa.kx = h->d_kx;
    fa.ky = h->d_ky;
    fa.info = k.info;
    fa.abr = k.abr;
    fa.rowflip = k.rowflip;
    fa.colflip = k.colflip;
    CK(cudaMemsetAsync(k.info, 0, (size_t)std::max(h->nact, 1) * sizeof(int), h->stream));
    if (k.real) launch_factor_real(fa, h->stream);
    else launch_factor(fa, h->stream);
    ++h->launches;
  }
  if (!h->zs.empty()) {
    ZeroArgs za{};
    za.nsys = (int)h->zs.size();
    for (size_t s = 0; s < h->zs.size(); ++s) za.sys[s] = h->zs[s].dev;
    za.zsca = zsca;
    za.info = h->zinfo;
    launch_zero_factor(za, h->stream);
    ++h->launches;
  }
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(h->stream));
  for (auto& k : h->ks) {
    std::vector<int> info(std::max(h->nact, 1));
    CK(cudaMemcpy(info.data(), k.info, info.size() * sizeof(int), cudaMemcpyDeviceToHost));
    for (int i = 0; i < h->nact; ++i)
      if (info[i]) throw CoralError(CORAL_ESINGULAR, "zero pivot in the factorisation of a (kx,ky) system");
  }
  if (!h->zs.empty()) {
    std::vector<int> info(kMaxSets);
    CK(cudaMemcpy(info.data(), h->zinfo, kMaxSets * sizeof(int), cudaMemcpyDeviceToHost));
    for (size_t s = 0; s < h->zs.size(); ++s)
      if (info[s]) throw CoralError(CORAL_ESINGULAR, "zero pivot in the factorisation of a mean system");
  }
  h->dt_factored = dt;
  if (h->graph) {
    cudaGraphExecDestroy(h->graph);
    h->graph = nullptr;
  }
}

void march(coral_handle* h, double dt, int nsteps) {
  if (!(dt > 0.0) || nsteps < 0) throw CoralError(CORAL_EBADARG, "march: dt must be > 0 and nsteps >= 0");
  if (!h->src_missing.empty()) throw CoralError(CORAL_EBADARG, h->src_missing);
  CK(cudaSetDevice(h->device));
  if (h->dt_factored != dt) factorize(h, dt);
  int done = 0;
  if (!h->graph || h->graph_dt != dt) {
    // one eager step (sets kernel attributes), then capture one step as a graph
    if (nsteps == 0) return;
    h->launches_per_step = enqueue_step(h, dt);
    h->launches += h->launches_per_step;
    done = 1;
    if (h->graph) {
      cudaGraphExecDestroy(h->graph);
      h->graph = nullptr;
    }
    cudaGraph_t gr;
    CK(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    try {
      enqueue_step(h, dt);
    } catch (...) {
      cudaStreamEndCapture(h->stream, &gr);
      throw;
    }
    CK(cudaStreamEndCapture(h->stream, &gr));
    CK(cudaGraphInstantiate(&h->graph, gr, 0));
    cudaGraphDestroy(gr);
    h->graph_dt = dt;
  }
  for (int s = done; s < nsteps; ++s) {
    CK(cudaGraphLaunch(h->graph, h->stream));
    h->launches += h->launches_per_step;
  }
}

void check_sys(coral_handle* h, int isys, bool zero) {
  if (isys < 0 || isys >= (int)(zero ? h->zs.size() : h->ks.size()))
    throw CoralError(CORAL_EBADARG, "system index out of range");
}

void spec_to_phys_dev(coral_handle* h, const double2* d_spec, double* d_phys_out) {
  const Dims& d = h->d;
  launch_inv_y(d, 1, h->d_fv, StateSet{}, d_spec, h->d_kx, h->d_ky, h->Y1, h->py, h->stream);
  launch_inv_x(d, 1, h->Y1, h->Y2, h->px, h->stream);
  launch_inv_z(d, 1, h->Y2, d_phys_out, h->pz, h->dct_tw, h->d_wz, nullptr, h->stream);
  h->launches += 3;
}

void phys_to_spec_dev(coral_handle* h, const double* d_phys, double2* d_spec_out) {
  const Dims& d = h->d;
  const Geometry& g = *h->G;
  QuadDesc q{};
  q.nq = 1;
  q.v1[0] = 0;
  q.v2[0] = -1;
  q.ke_q[0] = q.ke_q[1] = q.ke_q[2] = -1;
  launch_fwd_z(d, 1, q, d_phys, h->Y2, h->pz, h->dct_tw, h->d_wz, nullptr, h->stream);
  launch_fwd_x(d, 1, h->Y2, h->Y1, h->px, h->stream);
  launch_fwd_y(d, 1, h->Y1, d_spec_out, 1.0 / ((double)g.NXAA * g.NYAA * g.NZAA), h->py, h->stream);
  h->launches += 3;
}

std::vector<double> read_file(const std::string& fn, size_t n) {
  std::vector<double> v(n);
  FILE* f = std::fopen(fn.c_str(), "rb");
  if (!f) throw CoralError(CORAL_EIO, "cannot open " + fn);
  size_t r = std::fread(v.data(), sizeof(double), n, f);
  std::fclose(f);
  if (r != n) throw CoralError(CORAL_EIO, "short read in " + fn);
  return v;
}

void write_file(const std::string& fn, const std::vector<double>& v) {
  FILE* f = std::fopen(fn.c_str(), "wb");
  if (!f) throw CoralError(CORAL_EIO, "cannot create " + fn);
  size_t w = std::fwrite(v.data(), sizeof(double), v.size(), f);
  std::fclose(f);
  if (w != v.size()) throw CoralError(CORAL_EIO, "short write in " + fn);
}

std::string qs_name(const char* dir, const char* kind, int sys, int var, int rolling) {
  char b[96];
  std::snprintf(b, sizeof(b), "/QuickSave.%s.sys%03d.var%03d.rolling%d", kind, sys, var, rolling);
  return std::string(dir) + b;
}

// one coupled variable from a physical field already on the device ([y][x][z])
void set_var_phys_dev(coral_handle* h, int s, int v, const double* d_phys) {
  KSys& k = h->ks[s];
  const Dims& d = h->d;
  phys_to_spec_dev(h, d_phys, h->tmp_spec);
  // clear the variable's slots, then insert its projection
  std::vector<int> zero_slots = k.ops.var_pos[v];
  (void)zero_slots;
  launch_galerkin_insert(d, h->tmp_spec, k.T, k.d_var_pos[v], k.ops.var_size[v], k.d_sq_val[v], k.d_sq_col[v],
                         k.field, h->stream);
  h->launches += 1;
  CK(cudaGetLastError());
}

// mean-profile (NZAA values) <-> Galerkin coefficients of one mean variable, via
// the (0,0) column of the 3-D transforms
void import_zero_var(coral_handle* h, ZSys& z, int v, const std::vector<double>& prof) {
  const Geometry& g = *h->G;
  std::vector<double> phys((size_t)g.NYAA * g.NXAA * g.NZAA);
  for (size_t c = 0; c < (size_t)g.NYAA * g.NXAA; ++c)
    std::memcpy(&phys[c * g.NZAA], prof.data(), g.NZAA * sizeof(double));
  CK(cudaMemcpyAsync(h->tmp_phys, phys.data(), phys.size() * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  phys_to_spec_dev(h, h->tmp_phys, h->tmp_spec);
  std::vector<double2> cheb(g.NZ);
  CK(cudaMemcpyAsync(cheb.data(), h->tmp_spec, g.NZ * sizeof(double2), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  // forward substitution with the (lower-triangular) square stencil
  const SystemOps& o = z.ops;
  const int nc = o.var_size[v];
  std::vector<double> gal(nc, 0.0);
  for (int r = 0; r < nc; ++r) {
    double acc = cheb[r].x, diag = 1.0;
    for (auto& e : o.stencil_rows[v][r]) {
      if (e.first == r) diag = e.second;
      else if (e.first < r) acc -= e.second * gal[e.first];
    }
    gal[r] = acc / diag;
  }
  std::vector<double> field(o.T);
  CK(cudaMemcpy(field.data(), z.dev.field, o.T * sizeof(double), cudaMemcpyDeviceToHost));
  for (int c = 0; c < nc; ++c) field[o.var_pos[v][c]] = gal[c];
  CK(cudaMemcpy(z.dev.field, field.data(), o.T * sizeof(double), cudaMemcpyHostToDevice));
}

std::vector<double> export_zero_var(coral_handle* h, ZSys& z, int v) {
  const Geometry& g = *h->G;
  const size_t nsys = (size_t)g.NXH * g.NYAA;
  std::vector<double> field(z.ops.T);
  CK(cudaMemcpy(field.data(), z.dev.field, z.ops.T * sizeof(double), cudaMemcpyDeviceToHost));
  std::vector<double2> spec(nsys * g.NZ, make_double2(0.0, 0.0));
  for (int n = 0; n < g.NZ; ++n) {
    double s = 0.0;
    for (int k = 0; k < kTabW; ++k) {
      int tt = z.tab_t[v][(size_t)n * kTabW + k];
      if (tt >= 0) s += z.tab_v[v][(size_t)n * kTabW + k] * field[tt];
    }
    spec[n] = make_double2(s, 0.0);
  }
  CK(cudaMemcpyAsync(h->tmp_spec, spec.data(), spec.size() * sizeof(double2), cudaMemcpyHostToDevice, h->stream));
  spec_to_phys_dev(h, h->tmp_spec, h->tmp_phys);
  std::vector<double> prof(g.NZAA);
  CK(cudaMemcpyAsync(prof.data(), h->tmp_phys, g.NZAA * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return prof;
}

// mkdir -p
int mkdir_p(const std::string& path) {
  std::string cur;
  for (size_t i = 0; i <= path.size(); ++i) {
    if (i == path.size() || path[i] == '/') {
      if (!cur.empty() && ::mkdir(cur.c_str(), 0755) != 0 && errno != EEXIST) return -1;
    }
    if (i < path.size()) cur.push_back(path[i]);
  }
  return 0;
}

// cargo%cfl_based_DT from the CFL maxima of the last step's last stage
// (compute_cfl_based_timestep, marching.f90:219-251): the w term scaled by
// cflFactor_along_z (skipped at or below 1e-10), and with the Smagorinsky
// viscosity the diffusive limit 0.95 / ((2 pi)^2 max(nuSmago) (dx^-2 + dy^-2)),
// whose literals 0.95 and 3.141592 are single precision there
double cfl_dt_of(const coral_handle* h, const unsigned long long bits[4]) {
  const Geometry& g = *h->G;
  double mx[4];
  for (int i = 0; i < 4; ++i) std::memcpy(&mx[i], &bits[i], sizeof(double));
  const double u = mx[0] * g.NXAA / g.Lx, v = mx[1] * g.NYAA / g.Ly;
  const double w = h->cfl_factor_z > 1e-10 ? std::max(v, mx[2] * h->cfl_factor_z) : v;
  const double m = std::max(u, std::max(v, w));
  double cfl = (h->nF >= 3 && m > 0.0) ? 1.0 / m : (h->nF >= 3 ? INFINITY : 1.0);
  if (h->smago_var >= 0) {
    const float tp = 2.0f * 3.141592f;
    const double den = (double)(tp * tp) * mx[3] *
                       ((g.NXAA / g.Lx) * (g.NXAA / g.Lx) + (g.NYAA / g.Ly) * (g.NYAA / g.Ly));
    if (den > 0.0) cfl = std::min(cfl, (double)0.95f / den);
  }
  return cfl;
}

std::string trim(const std::string& t) {
  size_t a = t.find_first_not_of(" \t\r\n"), b = t.find_last_not_of(" \t\r\n");
  return a == std::string::npos ? std::string() : t.substr(a, b - a + 1);
}

// coral.timeseries (master_recipe%add_timeseries, PL_equations.f90:233-320 with
// get_timeseriesVarName_period[_position], PL_string_to_data.f90:200-242):
//   >>Volume_average :: NAME <<
//   >>Horizontal_avg :: NAME ;; Position= K <<      (K: 1-based z grid index)
// until >>EOF<<.  Positions beyond NZAA are ignored (as the reference does);
// NAME is a full variable or a quadratic variable.  Objects are ordered as the
// reference fills its buffer: full variables in recipe order, then quadratic
// variables, each with its objects in file order.
void set_timeseries(coral_handle* h, const std::string& text) {
  struct Obj { int src, z; std::string file; };
  std::vector<std::vector<Obj>> per_full(h->nF), per_quad(h->nQ);
  std::istringstream in(text);
  std::string line;
  const int NZAA = h->G->NZAA;
  while (std::getline(in, line)) {
    if (line.size() >= 5 && line.compare(2, 3, "EOF") == 0) break;
    if (trim(line).empty()) continue;
    const std::string head = line.substr(0, std::min<size_t>(19, line.size()));
    const size_t dc = line.find("::"), end = line.find("<<", 2);
    if (dc == std::string::npos || end == std::string::npos || end < dc)
      throw CoralError(CORAL_EPARSE, "coral.timeseries: cannot read line '" + line + "'");
    std::string name;
    int zpos = -1;
    if (head == ">>Volume_average ::") {
      name = trim(line.substr(dc + 2, end - dc - 2));
    } else if (head == ">>Horizontal_avg ::") {
      const size_t pp = line.find(";; Position=");
      if (pp == std::string::npos || pp < dc)
        throw CoralError(CORAL_EPARSE, "coral.timeseries: no ';; Position=' in '" + line + "'");
      name = trim(line.substr(dc + 2, pp - dc - 2));
      zpos = std::atoi(trim(line.substr(pp + 12, end - pp - 12)).c_str());
      if (zpos > NZAA) continue;  // ignored, as by the reference
      if (zpos < 1) throw CoralError(CORAL_EPARSE, "coral.timeseries: position must be >= 1 in '" + line + "'");
    } else {
      throw CoralError(CORAL_EPARSE, "coral.timeseries: lines must start with '>>Volume_average ::' or "
                                     "'>>Horizontal_avg ::' ('" + line + "')");
    }
    char ext[32];
    if (zpos < 0) std::snprintf(ext, sizeof(ext), "_volAvg.dat");
    else std::snprintf(ext, sizeof(ext), "_XYavg_z%05d.dat", zpos);
    for (int f = 0; f < h->nF; ++f)
      if (h->R.full[f].name == name) per_full[f].push_back({f, zpos - 1, name + ext});
    for (int q = 0; q < h->nQ; ++q)
      if (h->R.quad[q].name == name) per_quad[q].push_back({-1 - q, zpos - 1, name + ext});
  }
  std::vector<Obj> all;
  for (auto& v : per_full) all.insert(all.end(), v.begin(), v.end());
  for (auto& v : per_quad) all.insert(all.end(), v.begin(), v.end());
  if (all.size() > (size_t)kMaxTs)
    throw CoralError(CORAL_EUNSUPPORTED, "coral.timeseries: more than " + std::to_string(kMaxTs) + " objects");
  h->quads.ts_n = (int)all.size();
  h->ts_file.clear();
  for (size_t o = 0; o < all.size(); ++o) {
    h->quads.ts_src[o] = all[o].src;
    h->quads.ts_z[o] = all[o].z;
    h->ts_file.push_back(all[o].file);
  }
  // the step graph bakes in the objects: capture it again
  if (h->graph) {
    cudaGraphExecDestroy(h->graph);
    h->graph = nullptr;
  }
  h->ts_rows.clear();
}

// Append the buffered timeseries rows to <dir>/Timeseries/*.dat: raw float64,
// the value of step k at byte offset 8 (k - 1), a file started afresh when
// step 1 is written (output_2Dbundled_dsca_in_unique_timeserie calls of
// PL_IMEX_timestepping_output.f90:136-231).
void flush_timeseries(coral_handle* h, const std::string& dir) {
  if (h->ts_rows.empty()) return;
  const std::string tsdir = dir + "/Timeseries";
  FILE* probe = std::fopen((tsdir + "/.").c_str(), "rb");
  if (probe) std::fclose(probe);
  else if (mkdir_p(tsdir) != 0) throw CoralError(CORAL_EIO, "cannot create " + tsdir);
  const int n = h->quads.ts_n;
  for (int o = -1; o < n; ++o) {  // -1: time.dat
    const std::string fn = tsdir + "/" + (o < 0 ? std::string("time.dat") : h->ts_file[o]);
    const long long first = h->ts_rows.front().first;
    FILE* f = std::fopen(fn.c_str(), first == 1 ? "wb" : "r+b");
    if (!f) f = std::fopen(fn.c_str(), "wb");
    if (!f) throw CoralError(CORAL_EIO, "cannot open " + fn);
    std::vector<double> col;
    col.reserve(h->ts_rows.size());
    for (auto& r : h->ts_rows) col.push_back(r.second[o + 1]);
    if (std::fseek(f, (long)((first - 1) * 8), SEEK_SET) != 0 ||
        std::fwrite(col.data(), sizeof(double), col.size(), f) != col.size()) {
      std::fclose(f);
      throw CoralError(CORAL_EIO, "short write in " + fn);
    }
    std::fclose(f);
  }
  h->ts_rows.clear();
}

// initialise_bookkeeping_counters (PL_IMEX_timestepping_marching.f90:620-637)
void usr_output_counters(coral_handle* h) {
  h->time_integer = h->i_timestep;
  for (auto& o : h->uo) o.counter = h->i_timestep % o.period;
}

// add_outputs (PL_equations.f90:322-427) with the line readers of
// PL_string_to_data.f90:244-300: '>>Volume :: var ;; Period= N <<',
// '>>XSlice ::' / '>>YSlice ::' / '>>ZSlice ::' with ';; Position= I' (ignored
// beyond NXAA / NYAA / NZAA), '>>Zsummed::', '>>Profile::'; objects kept per
// variable, full variables first, each in file order.
void set_usr_output(coral_handle* h, const std::string& text) {
  std::vector<std::vector<coral_handle::UsrOut>> per_full(h->nF), per_quad(h->nQ);
  std::istringstream in(text);
  std::string line;
  const Geometry& g = *h->G;
  while (std::getline(in, line)) {
    if (line.size() >= 5 && line.compare(2, 3, "EOF") == 0) break;
    if (trim(line).empty()) continue;
    const std::string head = line.substr(0, std::min<size_t>(11, line.size()));
    int kind = -1, limit = 0;
    if (head == ">>Volume ::") kind = 0;
    else if (head == ">>ZSlice ::") kind = 1, limit = g.NZAA;
    else if (head == ">>YSlice ::") kind = 2, limit = g.NYAA;
    else if (head == ">>XSlice ::") kind = 3, limit = g.NXAA;
    else if (head == ">>Zsummed::") kind = 4;
    else if (head == ">>Profile::") kind = 5;
    else
      throw CoralError(CORAL_EPARSE, "coral.usrOutput: lines must start with '>>Volume ::', '>>XSlice ::', "
                                     "'>>YSlice ::', '>>ZSlice ::', '>>Profile::' or '>>Zsummed::' ('" + line + "')");
    const size_t dc = line.find("::"), pp = line.find(";; Period="), end = line.find("<<");
    const size_t ps = line.find(";; Position=");
    const bool positioned = kind >= 1 && kind <= 3;
    if (dc == std::string::npos || pp == std::string::npos || end == std::string::npos || pp < dc || end < pp ||
        (positioned && (ps == std::string::npos || ps < pp || end < ps)))
      throw CoralError(CORAL_EPARSE, "coral.usrOutput: cannot read line '" + line + "'");
    const std::string name = trim(line.substr(dc + 2, pp - dc - 2));
    const long long period = std::atoll(trim(line.substr(pp + 10, (positioned ? ps : end) - pp - 10)).c_str());
    int pos = 0;
    if (positioned) {
      pos = std::atoi(trim(line.substr(ps + 12, end - ps - 12)).c_str());
      if (pos > limit) continue;  // ignored, as by the reference
      if (pos < 1) throw CoralError(CORAL_EPARSE, "coral.usrOutput: position must be >= 1 in '" + line + "'");
    }
    if (period < 1) throw CoralError(CORAL_EPARSE, "coral.usrOutput: period must be >= 1 in '" + line + "'");
    for (int f = 0; f < h->nF; ++f)
      if (h->R.full[f].name == name) per_full[f].push_back({kind, f, pos - 1, period, 0});
    for (int q = 0; q < h->nQ; ++q)
      if (h->R.quad[q].name == name) {
        // output_slices_volumes_and_profiles has no vertically summed slice of a
        // quadratic variable (it stops with an error there)
        if (kind == 4) throw CoralError(CORAL_EUNSUPPORTED, "coral.usrOutput: no Zsummed output of a quadratic variable");
        per_quad[q].push_back({kind, -1 - q, pos - 1, period, 0});
      }
  }
  h->uo.clear();
  for (auto& v : per_full) h->uo.insert(h->uo.end(), v.begin(), v.end());
  for (auto& v : per_quad) h->uo.insert(h->uo.end(), v.begin(), v.end());
  usr_output_counters(h);
  if (!h->uo.empty() && !h->uo_buf) h->uo_buf = h->mem.get<double>((size_t)g.NYAA * g.NXAA * g.NZAA);
}

// The physical field of output source src from the current state; the full
// variables must be in fphys (full_vars_to_phys).  A quadratic variable is the
// product (compute_NL_terms_to_K_hat, marching.f90:279-291), with its vertical
// mean removed through its spectrum when the recipe asks (:292-298).
const double* usr_field(coral_handle* h, int src) {
  const Dims& d = h->d;
  const size_t np = (size_t)d.NYA * d.NXA * d.NZA;
  if (src >= 0) return h->fphys + (size_t)src * np;
  const QuadVar& Q = h->R.quad[-1 - src];
  const double* a = h->fphys + (size_t)(Q.v1 < 0 ? Q.v2 : Q.v1) * np;
  const double* b = (Q.v1 < 0 || Q.v2 < 0) ? nullptr : h->fphys + (size_t)Q.v2 * np;
  launch_phys_product(np, a, b, h->tmp_phys, h->stream);
  ++h->launches;
  if (Q.remove_mean) {
    phys_to_spec_dev(h, h->tmp_phys, h->tmp_spec);
    launch_remove_zmean(d, h->tmp_spec, h->stream);
    spec_to_phys_dev(h, h->tmp_spec, h->tmp_phys);
    ++h->launches;
  }
  return h->tmp_phys;
}

// export_volume / export_slice / export_verticallyAvgedSlice / export_profile
// (PL_IMEX_timestepping_output.f90:250-307,489-581,685-715): the file under dir,
// raw float64 in the reference's order, replaced if it exists.
void write_usr_object(coral_handle* h, const coral_handle::UsrOut& o, long long itime, const std::string& dir) {
  const Dims& d = h->d;
  const double* f = usr_field(h, o.src);
  const bool lin = o.src >= 0;
  const int iv = lin ? o.src + 1 : -o.src;
  const char* pre = lin ? "linear" : "quadra";
  char name[160];
  const char* sub = "Slices";
  size_t n = 0;
  double* out = h->uo_buf;
  if (!h->writer) {
    h->writer = std::make_unique<OutputWriter>();
    h->writer->start(h->device);
  }
  h->writer->order(h->stream);  // the previous object's copy out of uo_buf
  switch (o.kind) {
    case 0:
      sub = "Volumes";
      std::snprintf(name, sizeof(name), "%s_var%02d_time%08lld_full.dat", pre, iv, itime);
      launch_transpose_xy(d, f, out, 1, h->stream);
      n = (size_t)d.NXA * d.NYA * d.NZA;
      break;
    case 1: case 2: case 3: {
      const char axis = o.kind == 1 ? 'z' : (o.kind == 2 ? 'y' : 'x');
      std::snprintf(name, sizeof(name), "%s_var%02d_%c%05d_time%08lld_full.dat", pre, iv, axis, o.index + 1, itime);
      launch_usr_slice(d, f, o.kind, o.index, h->d_wz, out, h->stream);
      n = o.kind == 1 ? (size_t)d.NXA * d.NYA : (o.kind == 2 ? (size_t)d.NXA * d.NZA : (size_t)d.NYA * d.NZA);
      break;
    }
    case 4:
      std::snprintf(name, sizeof(name), "%s_var%02d_zAvged_time%08lld_full.dat", pre, iv, itime);
      launch_usr_slice(d, f, 4, 0, h->d_wz, out, h->stream);
      n = (size_t)d.NXA * d.NYA;
      break;
    default:
      sub = "Profiles";
      std::snprintf(name, sizeof(name), "%s_var%02d_time%08lld_full.dat", pre, iv, itime);
      launch_usr_profile(d, f, out, h->stream);
      n = d.NZA;
  }
  ++h->launches;
  CK(cudaGetLastError());
  const std::string sdir = dir + "/" + sub;
  h->writer->submit(out, n, h->stream, sdir, sdir + "/" + name);
}

// output_slices_volumes_and_profiles (PL_IMEX_timestepping_marching.f90:639-697),
// at the first stage of a step, i.e. from the state at its start: time_integer
// and every object's counter advance, the objects whose counter reaches their
// period are written (dir null: counters only).
void usr_output_step(coral_handle* h, const char* dir) {
  ++h->time_integer;
  std::vector<const coral_handle::UsrOut*> due;
  for (auto& o : h->uo)
    if (++o.counter == o.period) {
      o.counter = 0;
      due.push_back(&o);
    }
  if (due.empty() || !dir) return;
  h->launches += full_vars_to_phys(h, true, false);
  for (auto* o : due) write_usr_object(h, *o, h->time_integer, dir);
}

// The time loop of plane_layer_main.f90:138-205 for nsteps steps, with the
// dt rules of timeKeeping.f90: after each step dt = CFL_C * cfl_based_DT
// capped at dt_max (compare_dt_against_CFL, :78-89; stop below dt_min = 1e-9);
// before each step, dt_current takes the target dt when they differ by more
// than tolerance * dt_current, and the operators are refactorised
// (update_dt_if_needed, :171-183; factorize_operators).  The timeseries
// objects are recorded every step (time at the start of the step and the
// values of its first stage) and written to <dir>/Timeseries every 20 steps
// (buffer_length, PL_IMEX_timestepping.f90:159) and at the end.
// A call that fails part way still waits for the files it queued, and their
// errors go with it (the next call starts clean).
struct DrainWriterOnThrow {
  coral_handle* h;
  bool done = false;
  ~DrainWriterOnThrow() {
    if (done || !h->writer) return;
    try {
      h->writer->flush();
    } catch (const CoralError&) {
    }
  }
};

void run_loop(coral_handle* h, int nsteps, const char* outdir) {
  DrainWriterOnThrow drain{h};
  if (nsteps < 0) throw CoralError(CORAL_EBADARG, "coral_run: nsteps must be >= 0");
  if (outdir && !*outdir) outdir = nullptr;  // an empty string (a Fortran c_null_char) means no output
  const Parameters& P = h->P;
  const double dt_min = 1e-9;
  const int n = h->quads.ts_n;
  for (int s = 0; s < nsteps; ++s) {
    // check_for_update
    if (std::fabs(h->dt_target - h->dt_current) > P.tolerance * h->dt_current) {
      h->dt_current = h->dt_target;
      ++h->refactorizations;
    }
    if (!h->uo.empty()) usr_output_step(h, outdir);
    march(h, h->dt_current, 1);  // refactorises when dt_current changed
    CK(cudaMemcpyAsync(h->h_pin + kMaxTs, h->cfl_bits, 4 * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                       h->stream));
    if (n > 0)
      CK(cudaMemcpyAsync(h->h_pin, h->ts_out, n * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    if (n > 0 || outdir) {
      std::vector<double> row(n + 1);
      row[0] = h->time;
      for (int o = 0; o < n; ++o) row[o + 1] = h->h_pin[o];
      h->ts_rows.emplace_back(h->i_timestep, std::move(row));
    }
    unsigned long long bits[4];
    std::memcpy(bits, h->h_pin + kMaxTs, sizeof(bits));
    const double cfl = cfl_dt_of(h, bits);
    // apply_cfl
    double dt = cfl * P.CFL_C;
    if (!(dt <= P.dt_max)) dt = P.dt_max;  // also when cfl is infinite or NaN
    if (!(cfl == cfl)) throw CoralError(CORAL_ENONFINITE, "non-finite velocity maximum in the CFL criterion");
    if (dt < dt_min) throw CoralError(CORAL_ENONFINITE, "minimal timestep reached (dt < 1e-9)");
    h->dt_target = dt;
    // increment
    h->time += h->dt_current;
    ++h->i_timestep;
    if (outdir && h->ts_rows.size() >= 20) flush_timeseries(h, outdir);
  }
  if (outdir) flush_timeseries(h, outdir);
  else h->ts_rows.clear();
  drain.done = true;
  if (h->writer) h->writer->flush();  // the call's files are on disk when it returns
}

template <typename F>
int guarded(coral_handle* h, F&& f) {
  if (!h) return CORAL_EBADARG;
  try {
    CK(cudaSetDevice(h->device));
    f();
    return CORAL_OK;
  } catch (const CoralError& e) {
    h->err = e.what();
    return e.code;
  } catch (const std::exception& e) {
    h->err = e.what();
    return CORAL_EBADARG;
  }
}

std::string slurp(const char* path) {
  std::ifstream f(path, std::ios::binary);
  if (!f) throw CoralError(CORAL_EIO, std::string("cannot open ") + path);
  std::stringstream ss;
  ss << f.rdbuf();
  return ss.str();
}

}  // namespace

extern "C" {

namespace {
// the y pipeline's side streams and events, created when the variant is first
// selected (outside any stream capture)
void ensure_ystreams(coral_handle* h) {
  if (h->yfork) return;
  for (int k = 0; k < kYStreams; ++k) {
    CK(cudaStreamCreateWithFlags(&h->ystream[k], cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&h->yjoin[k], cudaEventDisableTiming));
  }
  CK(cudaEventCreateWithFlags(&h->yfork, cudaEventDisableTiming));
}
void release_streams(coral_handle* h) {
  for (int k = 0; k < kYStreams; ++k) {
    if (h->ystream[k]) cudaStreamDestroy(h->ystream[k]);
    if (h->yjoin[k]) cudaEventDestroy(h->yjoin[k]);
    h->ystream[k] = nullptr;
    h->yjoin[k] = nullptr;
  }
  if (h->yfork) cudaEventDestroy(h->yfork);
  h->yfork = nullptr;
  if (h->stream) cudaStreamDestroy(h->stream);
  h->stream = nullptr;
}
}  // namespace

namespace {
// the reference's command-line switches this library takes (plane_layer_main.f90:82;
// PL_IMEX_timestepping.f90:526-552); values are read as Fortran reals
int parse_args(const char* args, coral_handle* h) {
  if (!args) return CORAL_OK;
  std::istringstream is(args);
  std::vector<std::string> tok;
  std::string t;
  while (is >> t) tok.push_back(t);
  for (size_t i = 0; i < tok.size(); ++i) {
    auto value = [&](double* v) {
      if (i + 1 >= tok.size()) throw CoralError(CORAL_EBADARG, tok[i] + " needs a value");
      std::string x = tok[++i];
      for (char& c : x)
        if (c == 'd' || c == 'D') c = 'e';
      char* end = nullptr;
      *v = std::strtod(x.c_str(), &end);
      if (end == x.c_str() || *end) throw CoralError(CORAL_EBADARG, "bad value for " + tok[i - 1] + ": " + tok[i]);
    };
    if (tok[i] == "--withHorizontalSmagorinsky") h->smagorinsky = true;
    else if (tok[i] == "--smagorinsky-prefactor") value(&h->smago_prefactor);
    else if (tok[i] == "--cflFactor-along-z") value(&h->cfl_factor_z);
    else throw CoralError(CORAL_EBADARG, "unsupported argument: " + tok[i]);
  }
  return CORAL_OK;
}
}  // namespace

int coral_create(const char* equations_text, const char* parameters_text, const char* scheme, int device,
                 coral_handle** out) {
  return coral_create_with_args(equations_text, parameters_text, scheme, device, nullptr, out);
}

int coral_create_with_args(const char* equations_text, const char* parameters_text, const char* scheme, int device,
                           const char* args, coral_handle** out) {
  if (!out || !equations_text || !parameters_text) {
    g_create_error = "coral_create: null argument";
    return CORAL_EBADARG;
  }
  *out = nullptr;
  auto* h = new coral_handle();
  try {
    parse_args(args, h);
    setup(h, equations_text, parameters_text, scheme, device);
  } catch (const CoralError& e) {
    g_create_error = e.what();
    h->mem.free_all();
    if (h->h_pin) cudaFreeHost(h->h_pin);
    release_streams(h);
    delete h;
    return e.code;
  } catch (const std::exception& e) {
    g_create_error = e.what();
    h->mem.free_all();
    if (h->h_pin) cudaFreeHost(h->h_pin);
    release_streams(h);
    delete h;
    return CORAL_EBADARG;
  }
  *out = h;
  return CORAL_OK;
}

int coral_create_from_files(const char* equations_path, const char* parameters_path, const char* scheme, int device,
                            coral_handle** out) {
  if (!equations_path || !parameters_path) {
    g_create_error = "coral_create_from_files: null path";
    return CORAL_EBADARG;
  }
  std::string e, p;
  try {
    e = slurp(equations_path);
    p = slurp(parameters_path);
  } catch (const CoralError& err) {
    g_create_error = err.what();
    return err.code;
  }
  return coral_create(e.c_str(), p.c_str(), scheme, device, out);
}

void coral_destroy(coral_handle* h) {
  if (!h) return;
  cudaSetDevice(h->device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  if (h->writer) {
    try {
      h->writer->flush();
    } catch (const CoralError&) {
    }
    h->writer.reset();
  }
  if (h->graph) cudaGraphExecDestroy(h->graph);
  h->mem.free_all();
  if (h->h_pin) cudaFreeHost(h->h_pin);
  release_streams(h);
  delete h;
}

const char* coral_last_error(const coral_handle* h) { return h ? h->err.c_str() : g_create_error.c_str(); }

int coral_query(const coral_handle* hc, int what, long long* value) {
  if (!hc || !value) return CORAL_EBADARG;
  const coral_handle* h = hc;
  const Geometry& g = *h->G;
  switch (what) {
    case CORAL_Q_NX: *value = g.NX; return 0;
    case CORAL_Q_NY: *value = g.NY; return 0;
    case CORAL_Q_NZ: *value = g.NZ; return 0;
    case CORAL_Q_NXAA: *value = g.NXAA; return 0;
    case CORAL_Q_NYAA: *value = g.NYAA; return 0;
    case CORAL_Q_NZAA: *value = g.NZAA; return 0;
    case CORAL_Q_N_KXKY_SYSTEMS: *value = (long long)h->ks.size(); return 0;
    case CORAL_Q_N_ZERO_SYSTEMS: *value = (long long)h->zs.size(); return 0;
    case CORAL_Q_N_FULL_VARS: *value = h->nF; return 0;
    case CORAL_Q_N_QUAD_VARS: *value = h->nQ; return 0;
    case CORAL_Q_STAGES: *value = h->TB.stages; return 0;
    case CORAL_Q_DEVICE_BYTES: *value = (long long)h->mem.bytes; return 0;
    case CORAL_Q_KERNEL_LAUNCHES: *value = h->launches; return 0;
    default: break;
  }
  int base = (what / 100) * 100, i = what % 100;
  if (base == CORAL_Q_SYS_T && i < (int)h->ks.size()) { *value = h->ks[i].T; return 0; }
  if (base == CORAL_Q_ZSYS_T && i < (int)h->zs.size()) { *value = h->zs[i].dev.T; return 0; }
  if (base == CORAL_Q_SYS_NVARS && i < (int)h->ks.size()) { *value = h->ks[i].ops.nV; return 0; }
  if (base == CORAL_Q_ZSYS_NVARS && i < (int)h->zs.size()) { *value = h->zs[i].ops.nV; return 0; }
  if (base == CORAL_Q_SYS_KL && i < (int)h->ks.size()) { *value = h->ks[i].kl; return 0; }
  if (base == CORAL_Q_SYS_KU && i < (int)h->ks.size()) { *value = h->ks[i].ku; return 0; }
  if (base == CORAL_Q_SYS_REAL && i < (int)h->ks.size()) { *value = h->ks[i].real ? 1 : 0; return 0; }
  if (base == CORAL_Q_SYS_CLASSES && i < (int)h->ks.size()) { *value = h->ks[i].ncls; return 0; }
  if (base == CORAL_Q_SYS_CLASS_T && i < (int)h->ks.size()) { *value = h->ks[i].Tc; return 0; }
  if (base == CORAL_Q_SYS_CLASS_KL && i < (int)h->ks.size()) { *value = h->ks[i].kl_s; return 0; }
  if (base == CORAL_Q_SYS_CLASS_KU && i < (int)h->ks.size()) { *value = h->ks[i].ku_s; return 0; }
  if (base == CORAL_Q_SYS_FACTOR_ENTRIES && i < (int)h->ks.size()) {
    const KSys& k = h->ks[i];
    *value = 0;
    if (!k.lmask || h->dt_factored < 0.0) return 0;
    std::vector<unsigned> lm(k.Tc), um(k.Tc);
    if (cudaSetDevice(h->device) != cudaSuccess || cudaStreamSynchronize(h->stream) != cudaSuccess ||
        cudaMemcpy(lm.data(), k.lmask, k.Tc * sizeof(unsigned), cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(um.data(), k.umask, k.Tc * sizeof(unsigned), cudaMemcpyDeviceToHost) != cudaSuccess)
      return CORAL_ECUDA;
    long long n = 0;
    for (int j = 0; j < k.Tc; ++j) n += 1 + __builtin_popcount(lm[j]) + __builtin_popcount(um[j]);
    *value = n;
    return 0;
  }
  return CORAL_EBADARG;
}

int coral_factorize(coral_handle* h, double dt) {
  return guarded(h, [&] {
    if (!(dt > 0.0)) throw CoralError(CORAL_EBADARG, "dt must be > 0");
    factorize(h, dt);
  });
}

int coral_march(coral_handle* h, double dt, int nsteps) { return guarded(h, [&] { march(h, dt, nsteps); }); }

int coral_synchronize(coral_handle* h) {
  return guarded(h, [&] {
    CK(cudaStreamSynchronize(h->stream));
    unsigned int f = 0;
    CK(cudaMemcpy(&f, h->flags, sizeof(f), cudaMemcpyDeviceToHost));
    if (f & 2u) throw CoralError(CORAL_ECUDA, "a tensor-core wait of the z transform timed out");
    if (f & 1u) throw CoralError(CORAL_ENONFINITE, "non-finite value in the state");
  });
}

int coral_get_field(coral_handle* h, int isys, double* field) {
  return guarded(h, [&] {
    check_sys(h, isys, false);
    if (!field) throw CoralError(CORAL_EBADARG, "null buffer");
    const KSys& k = h->ks[isys];
    size_t n = (size_t)h->d.NXH * h->d.NYA * k.T;
    CK(cudaMemcpyAsync(field, k.field, n * sizeof(double2), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
  });
}

int coral_set_field(coral_handle* h, int isys, const double* field) {
  return guarded(h, [&] {
    check_sys(h, isys, false);
    if (!field) throw CoralError(CORAL_EBADARG, "null buffer");
    const KSys& k = h->ks[isys];
    size_t n = (size_t)h->d.NXH * h->d.NYA * k.T;
    CK(cudaMemcpyAsync(k.field, field, n * sizeof(double2), cudaMemcpyHostToDevice, h->stream));
    CK(cudaStreamSynchronize(h->stream));
  });
}

int coral_get_mean_field(coral_handle* h, int isys, double* field) {
  return guarded(h, [&] {
    check_sys(h, isys, true);
    if (!field) throw CoralError(CORAL_EBADARG, "null buffer");
    const ZSys& z = h->zs[isys];
    CK(cudaMemcpyAsync(field, z.dev.field, z.dev.T * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
  });
}

int coral_set_mean_field(coral_handle* h, int isys, const double* field) {
  return guarded(h, [&] {
    check_sys(h, isys, true);
    if (!field) throw CoralError(CORAL_EBADARG, "null buffer");
    const ZSys& z = h->zs[isys];
    CK(cudaMemcpyAsync(z.dev.field, field, z.dev.T * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    CK(cudaStreamSynchronize(h->stream));
  });
}

int coral_spec_to_phys(coral_handle* h, const double* spec, double* phys) {
  return guarded(h, [&] {
    if (!spec || !phys) throw CoralError(CORAL_EBADARG, "null buffer");
    const Dims& d = h->d;
    size_t ns = (size_t)d.NXH * d.NYA * d.NZ, np = (size_t)d.NYA * d.NXA * d.NZA;
    CK(cudaMemcpyAsync(h->tmp_spec, spec, ns * sizeof(double2), cudaMemcpyHostToDevice, h->stream));
    spec_to_phys_dev(h, h->tmp_spec, h->tmp_phys);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(phys, h->tmp_phys, np * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
  });
}

int coral_phys_to_spec(coral_handle* h, const double* phys, double* spec) {
  return guarded(h, [&] {
    if (!spec || !phys) throw CoralError(CORAL_EBADARG, "null buffer");
    const Dims& d = h->d;
    size_t ns = (size_t)d.NXH * d.NYA * d.NZ, np = (size_t)d.NYA * d.NXA * d.NZA;
    CK(cudaMemcpyAsync(h->tmp_phys, phys, np * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    phys_to_spec_dev(h, h->tmp_phys, h->tmp_spec);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(spec, h->tmp_spec, ns * sizeof(double2), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
  });
}

int coral_get_full_phys(coral_handle* h, int ivar, double* phys) {
  return guarded(h, [&] {
    if (ivar < 0 || ivar >= h->nF || !phys) throw CoralError(CORAL_EBADARG, "bad full-variable index or buffer");
    const Dims& d = h->d;
    h->launches += full_vars_to_phys(h, true, false);
    CK(cudaGetLastError());
    size_t np = (size_t)d.NYA * d.NXA * d.NZA;
    CK(cudaMemcpyAsync(phys, h->fphys + (size_t)ivar * np, np * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
  });
}

int coral_import_quicksave(coral_handle* h, const char* directory, int rolling) {
  return guarded(h, [&] {
    if (!directory) throw CoralError(CORAL_EBADARG, "null directory");
    const Dims& d = h->d;
    const size_t np = (size_t)d.NYA * d.NXA * d.NZA;
    for (size_t s = 0; s < h->ks.size(); ++s) {
      KSys& k = h->ks[s];
      CK(cudaMemsetAsync(k.field, 0, (size_t)d.NXH * d.NYA * k.T * sizeof(double2), h->stream));
      for (int v = 0; v < k.ops.nV; ++v) {
        std::vector<double> buf = read_file(qs_name(directory, "kxky", (int)s + 1, v + 1, rolling), np);
        CK(cudaMemcpyAsync(h->tmp_phys, buf.data(), np * sizeof(double), cudaMemcpyHostToDevice, h->stream));
        // file order is z fastest, then y, then x: transpose to (z, x, y)
        launch_transpose_xy(d, h->tmp_phys, h->fphys, 0, h->stream);
        h->launches += 1;
        set_var_phys_dev(h, (int)s, v, h->fphys);
        CK(cudaStreamSynchronize(h->stream));
      }
    }
    for (size_t s = 0; s < h->zs.size(); ++s) {
      ZSys& z = h->zs[s];
      CK(cudaMemset(z.dev.field, 0, z.dev.T * sizeof(double)));
      for (int v = 0; v < z.ops.nV; ++v)
        import_zero_var(h, z, v, read_file(qs_name(directory, "zero", (int)s + 1, v + 1, rolling), d.NZA));
    }
  });
}

int coral_export_checkpoint(coral_handle* h, const char* directory, int rolling) {
  return guarded(h, [&] {
    if (!directory) throw CoralError(CORAL_EBADARG, "null directory");
    const Dims& d = h->d;
    const size_t np = (size_t)d.NYA * d.NXA * d.NZA;
    std::vector<double> buf(np);
    for (size_t s = 0; s < h->ks.size(); ++s) {
      KSys& k = h->ks[s];
      for (int v = 0; v < k.ops.nV; ++v) {
        launch_cheb_extract(d, k.field, k.T, k.d_tab_t[v], k.d_tab_v[v], h->tmp_spec, h->stream);
        spec_to_phys_dev(h, h->tmp_spec, h->tmp_phys);
        launch_transpose_xy(d, h->tmp_phys, h->fphys, 1, h->stream);
        h->launches += 2;
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(buf.data(), h->fphys, np * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        write_file(qs_name(directory, "kxky", (int)s + 1, v + 1, rolling), buf);
        // as export_checkpoints does (PL_IMEX_timestepping_output.f90:412-425), the
        // variable's Galerkin coefficients are replaced by the projection of the
        // field just written (phys -> spec, square-stencil solve, insertion): the
        // state is then exactly what importing these files gives.  The other
        // variables' slots are untouched, so the next extraction reads the
        // original state; the mean systems are not re-projected (nor are they by
        // the reference).
        set_var_phys_dev(h, (int)s, v, h->tmp_phys);
      }
    }
    for (size_t s = 0; s < h->zs.size(); ++s)
      for (int v = 0; v < h->zs[s].ops.nV; ++v)
        write_file(qs_name(directory, "zero", (int)s + 1, v + 1, rolling), export_zero_var(h, h->zs[s], v));
  });
}

int coral_set_var_phys(coral_handle* h, int isys, int ivar, const double* phys) {
  return guarded(h, [&] {
    check_sys(h, isys, false);
    if (ivar < 0 || ivar >= h->ks[isys].ops.nV || !phys) throw CoralError(CORAL_EBADARG, "bad variable or buffer");
    const Dims& d = h->d;
    const size_t np = (size_t)d.NYA * d.NXA * d.NZA;
    CK(cudaMemcpyAsync(h->tmp_phys, phys, np * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    set_var_phys_dev(h, isys, ivar, h->tmp_phys);
    CK(cudaStreamSynchronize(h->stream));
  });
}

int coral_set_mean_var_profile(coral_handle* h, int isys, int ivar, const double* prof) {
  return guarded(h, [&] {
    check_sys(h, isys, true);
    if (ivar < 0 || ivar >= h->zs[isys].ops.nV || !prof) throw CoralError(CORAL_EBADARG, "bad variable or buffer");
    std::vector<double> p(prof, prof + h->d.NZA);
    import_zero_var(h, h->zs[isys], ivar, p);
  });
}

int coral_stream(coral_handle* h, void** stream) {
  return guarded(h, [&] {
    if (!stream) throw CoralError(CORAL_EBADARG, "null pointer");
    *stream = (void*)h->stream;
  });
}

int coral_profile_step(coral_handle* h, double dt, double* ms, int n) {
  return guarded(h, [&] {
    if (!ms || n < kProfileClasses) throw CoralError(CORAL_EBADARG, "need 11 timing slots");
    if (!(dt > 0.0)) throw CoralError(CORAL_EBADARG, "dt must be > 0");
    if (h->dt_factored != dt) factorize(h, dt);
    PhaseTimer pt{h->stream, {}};
    h->launches += enqueue_step(h, dt, &pt);
    CK(cudaStreamSynchronize(h->stream));
    for (int k = 0; k < n; ++k) ms[k] = 0.0;
    for (auto& e : pt.ev) {
      float t = 0.f;
      cudaEventElapsedTime(&t, e.second.first, e.second.second);
      ms[e.first] += t;
      cudaEventDestroy(e.second.first);
      cudaEventDestroy(e.second.second);
    }
  });
}

int coral_diagnostics(coral_handle* h, double* out3) {
  return guarded(h, [&] {
    if (!out3) throw CoralError(CORAL_EBADARG, "null buffer");
    const Geometry& g = *h->G;
    CK(cudaStreamSynchronize(h->stream));
    unsigned long long bits[4];
    CK(cudaMemcpy(bits, h->cfl_bits, sizeof(bits), cudaMemcpyDeviceToHost));
    out3[0] = cfl_dt_of(h, bits);
    // the partial sums are totalled on the device: 8 bytes come back, not the
    // per-CTA array
    if (h->zform_last == 1) launch_ke_sum(h->ke_partial_split, h->n_ke_split, h->ke_total, h->stream);
    else launch_ke_sum(h->ke_partial, h->n_ke_partial, h->ke_total, h->stream);
    ++h->launches;
    double ke = 0.0;
    CK(cudaMemcpyAsync(&ke, h->ke_total, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    out3[1] = ke / g.NXAA / g.NYAA;
    unsigned int f = 0;
    CK(cudaMemcpy(&f, h->flags, sizeof(f), cudaMemcpyDeviceToHost));
    out3[2] = (f & 1u) ? 1.0 : 0.0;
  });
}

int coral_set_timeseries(coral_handle* h, const char* timeseries_text) {
  return guarded(h, [&] {
    if (!timeseries_text) throw CoralError(CORAL_EBADARG, "null text");
    set_timeseries(h, timeseries_text);
  });
}

int coral_set_timeseries_from_file(coral_handle* h, const char* path) {
  return guarded(h, [&] {
    if (!path) throw CoralError(CORAL_EBADARG, "null path");
    set_timeseries(h, slurp(path));
  });
}

int coral_set_usr_output(coral_handle* h, const char* usr_output_text) {
  return guarded(h, [&] {
    if (!usr_output_text) throw CoralError(CORAL_EBADARG, "null text");
    set_usr_output(h, usr_output_text);
  });
}

int coral_set_usr_output_from_file(coral_handle* h, const char* path) {
  return guarded(h, [&] {
    if (!path) throw CoralError(CORAL_EBADARG, "null path");
    set_usr_output(h, slurp(path));
  });
}

int coral_export_usr_output(coral_handle* h, const char* output_directory, long long time_integer) {
  return guarded(h, [&] {
    if (!output_directory || !*output_directory) throw CoralError(CORAL_EBADARG, "null directory");
    if (h->uo.empty()) return;
    DrainWriterOnThrow drain{h};
    h->launches += full_vars_to_phys(h, true, false);
    for (auto& o : h->uo) write_usr_object(h, o, time_integer, output_directory);
    drain.done = true;
    h->writer->flush();
  });
}

int coral_timeseries(coral_handle* h, double* values, int n) {
  return guarded(h, [&] {
    const int m = h->quads.ts_n;
    if (n < m || (m > 0 && !values)) throw CoralError(CORAL_EBADARG, "buffer smaller than the timeseries objects");
    CK(cudaStreamSynchronize(h->stream));
    if (m > 0) CK(cudaMemcpy(values, h->ts_out, m * sizeof(double), cudaMemcpyDeviceToHost));
  });
}

int coral_set_time(coral_handle* h, double time, double dt, long long i_timestep) {
  return guarded(h, [&] {
    if (!(dt > 0.0) || i_timestep < 1) throw CoralError(CORAL_EBADARG, "dt must be > 0 and i_timestep >= 1");
    // read_timings_from_file (timeKeeping.f90:92-134) after its dt / 50: dt is
    // capped at dt_max
    const double d = dt <= h->P.dt_max ? dt : h->P.dt_max;
    h->time = time;
    h->dt_current = h->dt_target = d;
    h->i_timestep = i_timestep;
    h->ts_rows.clear();
    usr_output_counters(h);
  });
}

int coral_get_time(coral_handle* h, double* out4) {
  return guarded(h, [&] {
    if (!out4) throw CoralError(CORAL_EBADARG, "null buffer");
    out4[0] = h->time;
    out4[1] = h->dt_current;
    out4[2] = (double)h->i_timestep;
    out4[3] = (double)h->refactorizations;
  });
}

int coral_var_positions(coral_handle* h, int isys, int ivar, int* positions, int n, int* size) {
  return guarded(h, [&] {
    check_sys(h, isys, false);
    const SystemOps& o = h->ks[isys].ops;
    if (ivar < 0 || ivar >= o.nV) throw CoralError(CORAL_EBADARG, "variable index out of range");
    const auto& vp = o.var_pos[ivar];
    if (size) *size = (int)vp.size();
    if (!positions) return;
    if (n < (int)vp.size()) throw CoralError(CORAL_EBADARG, "buffer smaller than the variable");
    for (size_t i = 0; i < vp.size(); ++i) positions[i] = vp[i];
  });
}

namespace {
// the kernel variants of the step: name, the handle's switch, its default (a)
// and alternative (b) values with their names, and the timed phases they affect
struct Knob { const char* name; int* var; int a, b; const char* na; const char* nb; std::vector<int> phases; };
std::vector<Knob> knobs_of(coral_handle* h) {
  return {{"x_fft_plan", &h->tune.x_plan, 1, 0, "two-pass", "three-pass", {1, 4}},
          {"fwd_y_pass", &h->tune.fwd_y_grid, 0, 1, "persistent-pipelined", "one-CTA-per-tile", {5}},
          {"operator_tiles", &h->tune.generic_tiles, 0, 1, "compiled-groups", "run-time-forms", {7, 10}},
          {"band_substitution", &h->tune.subst_rt, 0, 1, "compiled-band", "run-time-band", {9}},
          {"z_pass", &h->tune.z_batch6, 1, 0, "6-line-batches", "9-line-batches", {3}},
          {"inv_y_pass", &h->tune.inv_y_loop, 0, 1, "single-term-build", "term-loop-build", {0}},
          {"inv_x_pass", &h->tune.inv_x_tiles, 1, 0, "one-CTA-per-tile", "persistent-pipelined", {1}},
          // timed over whole steps (its passes overlap across streams)
          {"y_pipeline", &h->tune.y_chunks, 1, 8, "whole-passes", "8-row-bands-3-streams", {-1}},
          // not timed by the autotuner (a factorisation, not a step phase)
          {"band_factor", &h->tune.factor_window, 1, 0, "shared-memory-window", "in-place", {}}};
}
}  // namespace

int coral_set_variant(coral_handle* h, const char* knob, int value) {
  return guarded(h, [&] {
    if (!knob) throw CoralError(CORAL_EBADARG, "set_variant: knob name is NULL");
    for (auto& kb : knobs_of(h)) {
      if (std::strcmp(kb.name, knob) != 0) continue;
      if (value != 0 && value != 1) throw CoralError(CORAL_EBADARG, "set_variant: value is 0 (default) or 1 (alternative)");
      if (kb.var == &h->tune.y_chunks) ensure_ystreams(h);
      *kb.var = value ? kb.b : kb.a;
      if (kb.var == &h->tune.factor_window && h->dt_factored >= 0.0) factorize(h, h->dt_factored);
      if (h->graph) {
        cudaGraphExecDestroy(h->graph);
        h->graph = nullptr;
      }
      return;
    }
    throw CoralError(CORAL_EBADARG, std::string("set_variant: unknown knob ") + knob);
  });
}

int coral_autotune(coral_handle* h, double dt, int repeats, char* report, int n) {
  return guarded(h, [&] {
    if (!(dt > 0.0) || repeats < 1) throw CoralError(CORAL_EBADARG, "autotune: dt > 0 and repeats >= 1");
    if (h->dt_factored != dt) factorize(h, dt);
    // the tuning steps advance a copy of the state: save it, restore it after
    std::vector<void*> saved;
    for (auto& k : h->ks) {
      void* p = nullptr;
      const size_t b = (size_t)h->d.NXH * h->d.NYA * k.T * sizeof(double2);
      CK(cudaMalloc(&p, b));
      CK(cudaMemcpyAsync(p, k.field, b, cudaMemcpyDeviceToDevice, h->stream));
      saved.push_back(p);
    }
    std::vector<std::vector<double>> zsaved;
    for (auto& z : h->zs) {
      std::vector<double> v(z.dev.T);
      CK(cudaMemcpy(v.data(), z.dev.field, z.dev.T * sizeof(double), cudaMemcpyDeviceToHost));
      zsaved.push_back(v);
    }
    // (the Smagorinsky viscosity carries from stage to stage: part of the state)
    std::vector<double> smago_saved;
    if (h->smago_prof) {
      smago_saved.resize(h->d.NZA);
      CK(cudaStreamSynchronize(h->stream));
      CK(cudaMemcpy(smago_saved.data(), h->smago_prof, h->d.NZA * sizeof(double), cudaMemcpyDeviceToHost));
    }
    auto time_phases = [&](std::initializer_list<int> phases) {
      double best = 1e300;
      for (int r = 0; r < repeats + 1; ++r) {  // the first step sets attributes and warms the caches
        PhaseTimer pt{h->stream, {}};
        enqueue_step(h, dt, &pt);
        CK(cudaStreamSynchronize(h->stream));
        double t = 0.0;
        for (auto& e : pt.ev) {
          float ms = 0.f;
          cudaEventElapsedTime(&ms, e.second.first, e.second.second);
          for (int ph : phases)
            if (e.first == ph) t += ms;
          cudaEventDestroy(e.second.first);
          cudaEventDestroy(e.second.second);
        }
        if (r > 0) best = std::min(best, t);
      }
      return best;
    };
    auto time_steps = [&]() {  // whole eager steps, CUDA events on the handle's stream
      double best = 1e300;
      cudaEvent_t a = nullptr, b = nullptr;
      CK(cudaEventCreate(&a));
      CK(cudaEventCreate(&b));
      for (int r = 0; r < repeats + 1; ++r) {
        CK(cudaEventRecord(a, h->stream));
        enqueue_step(h, dt, nullptr);
        CK(cudaEventRecord(b, h->stream));
        CK(cudaEventSynchronize(b));
        float ms = 0.f;
        cudaEventElapsedTime(&ms, a, b);
        if (r > 0) best = std::min(best, (double)ms);
      }
      cudaEventDestroy(a);
      cudaEventDestroy(b);
      return best;
    };
    ensure_ystreams(h);
    std::vector<Knob> knobs = knobs_of(h);
    std::string rep;
    for (auto& kb : knobs) {
      if (kb.phases.empty()) continue;
      auto timed = [&]() {
        if (kb.phases[0] < 0) return time_steps();
        if (kb.phases.size() == 2) return time_phases({kb.phases[0], kb.phases[1]});
        return time_phases({kb.phases[0]});
      };
      *kb.var = kb.a;
      const double ta = timed();
      *kb.var = kb.b;
      const double tb = timed();
      *kb.var = (tb < ta) ? kb.b : kb.a;
      char buf[256];
      std::snprintf(buf, sizeof(buf), "%s%s: %s %.4f ms, %s %.4f ms -> %s", rep.empty() ? "" : "; ", kb.name, kb.na, ta,
                    kb.nb, tb, (tb < ta) ? kb.nb : kb.na);
      rep += buf;
    }
    for (size_t i = 0; i < h->ks.size(); ++i) {
      const size_t b = (size_t)h->d.NXH * h->d.NYA * h->ks[i].T * sizeof(double2);
      CK(cudaMemcpyAsync(h->ks[i].field, saved[i], b, cudaMemcpyDeviceToDevice, h->stream));
    }
    CK(cudaStreamSynchronize(h->stream));
    for (void* p : saved) cudaFree(p);
    for (size_t i = 0; i < h->zs.size(); ++i)
      CK(cudaMemcpy(h->zs[i].dev.field, zsaved[i].data(), zsaved[i].size() * sizeof(double), cudaMemcpyHostToDevice));
    if (h->smago_prof)
      CK(cudaMemcpy(h->smago_prof, smago_saved.data(), h->d.NZA * sizeof(double), cudaMemcpyHostToDevice));
    if (h->graph) {
      cudaGraphExecDestroy(h->graph);
      h->graph = nullptr;
    }
    if (report && n > 0) {
      std::strncpy(report, rep.c_str(), (size_t)n - 1);
      report[n - 1] = 0;
    }
  });
}

int coral_closure_attach(coral_handle* h, coral_closure* c) {
  return guarded(h, [&] {
    if (c) {
      if (h->nF != 4 || h->nQ != 9)
        throw CoralError(CORAL_EUNSUPPORTED, "the closure needs 4 full variables (u, v, w, T) and 9 quadratic ones");
      if (h->zform != 0) throw CoralError(CORAL_EUNSUPPORTED, "the closure runs with the FP64 z transforms");
      if (!h->tau) h->tau = h->mem.get<double>((size_t)9 * h->d.NYA * h->d.NXA * h->d.NZA);
    }
    h->closure = c;
    if (h->graph) {
      cudaGraphExecDestroy(h->graph);
      h->graph = nullptr;
    }
  });
}

int coral_set_hermitian_kx0(coral_handle* h, int on) {
  return guarded(h, [&] {
    h->hermitian_kx0 = on != 0;
    if (h->graph) {
      cudaGraphExecDestroy(h->graph);
      h->graph = nullptr;
    }
  });
}

int coral_set_source(coral_handle* h, int index, const double* profile) {
  return guarded(h, [&] {
    if (!profile || index < 1 || index > 99) throw CoralError(CORAL_EBADARG, "source index must be 1..99");
    h->src_phys[index].assign(profile, profile + h->G->NZAA);
    update_sources(h);
  });
}

int coral_set_penalisation_mask(coral_handle* h, const double* mask) {
  return guarded(h, [&] {
    if (!mask) throw CoralError(CORAL_EBADARG, "null mask");
    if (std::none_of(h->R.full.begin(), h->R.full.end(), [](const FullVar& F) { return F.penal; }))
      throw CoralError(CORAL_EBADARG, "the recipe has no penalised variable");
    const size_t n = (size_t)h->d.NYA * h->d.NXA * h->d.NZA;
    CK(cudaStreamSynchronize(h->stream));
    CK(cudaMemcpy(h->tmp_phys, mask, n * sizeof(double), cudaMemcpyHostToDevice));
    penal_fields(h, h->tmp_phys);
  });
}

int coral_set_z_transform(coral_handle* h, int form) {
  return guarded(h, [&] { set_z_transform(h, form); });
}

int coral_run(coral_handle* h, int nsteps, const char* output_directory) {
  return guarded(h, [&] { run_loop(h, nsteps, output_directory); });
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Ensembles: many independent plane-layer runs (different grids, parameters
// and recipes) advanced together on one stream, one CUDA graph per step.  Per
// stage every member's transforms and right-hand sides are queued, then the
// band substitutions of all members run as one persistent launch
// (k_subst_tpb_multi), then every member's K_std and mean systems.  The
// reference solves its systems one (kx, ky) at a time in a loop
// (src/plane_layer/PL_algebra_z_3D.f90:197-214) and runs one problem per job.
// ---------------------------------------------------------------------------
struct coral_ensemble {
  std::string err;
  int device = 0;
  cudaStream_t stream = nullptr;
  std::vector<coral_handle*> mem;
  cudaGraphExec_t graph = nullptr;
  double graph_dt = -1.0;
  bool batched = false;                       // all members' substitutions in one launch
  std::vector<SolveArgs*> d_args;             // per stage: SolveArgs of every (member, system)
  std::vector<long long*> d_prefix;           // per stage: first block of each (member, system)
  std::vector<int> nsub;                      // per stage: (member, system) entries
  std::vector<long long> total;               // per stage: blocks in all
  long long launches = 0;
  int launches_per_step = 0;
  // members' own phases run on these streams (member m on stream m mod kEnsStreams),
  // forked from and joined back into `stream`: the step graph has one branch per stream
  std::vector<cudaStream_t> mstream;
  cudaEvent_t fork = nullptr;
  std::vector<cudaEvent_t> join;
};

namespace {

constexpr int kEnsStreams = 8;

// f(h) for every member, member m queued on member stream m mod kEnsStreams,
// forked from and joined back into the ensemble's stream
template <class F>
int ens_fan(coral_ensemble* e, F&& f) {
  int nl = 0;
  const int K = (int)e->mstream.size();
  CK(cudaEventRecord(e->fork, e->stream));
  for (int k = 0; k < K; ++k) CK(cudaStreamWaitEvent(e->mstream[k], e->fork, 0));
  for (size_t m = 0; m < e->mem.size(); ++m) {
    coral_handle* h = e->mem[m];
    h->stream = e->mstream[m % K];
    try {
      nl += f(h);
    } catch (...) {
      h->stream = e->stream;
      throw;
    }
    h->stream = e->stream;
  }
  for (int k = 0; k < K; ++k) {
    CK(cudaEventRecord(e->join[k], e->mstream[k]));
    CK(cudaStreamWaitEvent(e->stream, e->join[k], 0));
  }
  return nl;
}

void ens_free_args(coral_ensemble* e) {
  for (auto* p : e->d_args) cudaFree(p);
  for (auto* p : e->d_prefix) cudaFree(p);
  e->d_args.clear();
  e->d_prefix.clear();
  e->nsub.clear();
  e->total.clear();
}

// the per-stage argument tables of the batched substitution (for dt)
void ens_build_args(coral_ensemble* e, double dt) {
  ens_free_args(e);
  const int S = e->mem[0]->TB.stages;
  e->batched = true;
  for (int i = 0; i < S && e->batched; ++i) {
    std::vector<SolveArgs> args;
    std::vector<long long> prefix(1, 0);
    for (coral_handle* h : e->mem)
      for (auto& k : h->ks) {
        if (!k.real) { e->batched = false; break; }
        SolveArgs sa = make_solve_args(h, k, i, dt);
        if (!subst_multi_supported(sa)) { e->batched = false; break; }
        args.push_back(sa);
        prefix.push_back(prefix.back() + sa.nblk);
      }
    if (!e->batched) break;
    SolveArgs* da = nullptr;
    long long* dp = nullptr;
    CK(cudaMalloc(&da, args.size() * sizeof(SolveArgs)));
    e->d_args.push_back(da);
    CK(cudaMalloc(&dp, prefix.size() * sizeof(long long)));
    e->d_prefix.push_back(dp);
    CK(cudaMemcpy(da, args.data(), args.size() * sizeof(SolveArgs), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(dp, prefix.data(), prefix.size() * sizeof(long long), cudaMemcpyHostToDevice));
    e->nsub.push_back((int)args.size());
    e->total.push_back(prefix.back());
  }
  if (!e->batched) ens_free_args(e);
}

int ens_enqueue(coral_ensemble* e, double dt) {
  int nl = 0;
  const int S = e->mem[0]->TB.stages;
  for (int i = 0; i < S; ++i) {
    nl += ens_fan(e, [&](coral_handle* h) { return enqueue_stage_pre(h, i, dt, nullptr); });
    if (e->batched) {
      launch_subst_multi(e->d_args[i], e->d_prefix[i], e->nsub[i], e->total[i], e->stream);
      ++nl;
    } else {
      nl += ens_fan(e, [&](coral_handle* h) { return enqueue_stage_subst(h, i, dt, nullptr); });
    }
    nl += ens_fan(e, [&](coral_handle* h) { return enqueue_stage_post(h, i, dt, nullptr); });
  }
  nl += ens_fan(e, [&](coral_handle* h) { return enqueue_step_end(h); });
  CK(cudaGetLastError());
  return nl;
}

void ens_march(coral_ensemble* e, double dt, int nsteps) {
  if (!(dt > 0.0) || nsteps < 0) throw CoralError(CORAL_EBADARG, "march: dt must be > 0 and nsteps >= 0");
  CK(cudaSetDevice(e->device));
  bool refactored = false;
  for (coral_handle* h : e->mem)
    if (h->dt_factored != dt) {
      factorize(h, dt);
      refactored = true;
    }
  int done = 0;
  if (!e->graph || e->graph_dt != dt || refactored) {
    if (nsteps == 0) return;
    ens_build_args(e, dt);
    e->launches_per_step = ens_enqueue(e, dt);  // eager step (kernel attributes)
    e->launches += e->launches_per_step;
    done = 1;
    if (e->graph) {
      cudaGraphExecDestroy(e->graph);
      e->graph = nullptr;
    }
    cudaGraph_t gr;
    CK(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
    try {
      ens_enqueue(e, dt);
    } catch (...) {
      cudaStreamEndCapture(e->stream, &gr);
      throw;
    }
    CK(cudaStreamEndCapture(e->stream, &gr));
    CK(cudaGraphInstantiate(&e->graph, gr, 0));
    cudaGraphDestroy(gr);
    e->graph_dt = dt;
  }
  for (int s = done; s < nsteps; ++s) {
    CK(cudaGraphLaunch(e->graph, e->stream));
    e->launches += e->launches_per_step;
  }
}

template <typename F>
int ens_guarded(coral_ensemble* e, F&& f) {
  if (!e) return CORAL_EBADARG;
  try {
    CK(cudaSetDevice(e->device));
    f();
    return CORAL_OK;
  } catch (const CoralError& x) {
    e->err = x.what();
    return x.code;
  } catch (const std::exception& x) {
    e->err = x.what();
    return CORAL_EBADARG;
  }
}

void ens_destroy(coral_ensemble* e) {
  if (!e) return;
  cudaSetDevice(e->device);
  if (e->stream) cudaStreamSynchronize(e->stream);
  if (e->graph) cudaGraphExecDestroy(e->graph);
  ens_free_args(e);
  for (coral_handle* h : e->mem) {
    if (h->stream == e->stream) h->stream = nullptr;  // the ensemble's stream, destroyed below
    coral_destroy(h);
  }
  for (cudaStream_t st : e->mstream) cudaStreamDestroy(st);
  for (cudaEvent_t ev : e->join) cudaEventDestroy(ev);
  if (e->fork) cudaEventDestroy(e->fork);
  if (e->stream) cudaStreamDestroy(e->stream);
  delete e;
}

}  // namespace

extern "C" {

int coral_ensemble_create(int n, const char* const* equations_texts, const char* const* parameters_texts,
                          const char* scheme, int device, coral_ensemble** out) {
  if (!out || n <= 0 || !equations_texts || !parameters_texts) {
    g_create_error = "coral_ensemble_create: bad arguments";
    return CORAL_EBADARG;
  }
  *out = nullptr;
  auto* e = new coral_ensemble();
  e->device = device;
  for (int i = 0; i < n; ++i) {
    coral_handle* h = nullptr;
    const int rc = coral_create(equations_texts[i], parameters_texts[i], scheme, device, &h);
    if (rc != CORAL_OK) {
      const std::string msg = "member " + std::to_string(i) + ": " + g_create_error;
      ens_destroy(e);
      g_create_error = msg;
      return rc;
    }
    e->mem.push_back(h);
    if (h->TB.stages != e->mem[0]->TB.stages) {
      ens_destroy(e);
      g_create_error = "coral_ensemble_create: members use IMEX schemes with different stage counts";
      return CORAL_EBADARG;
    }
  }
  // the ensemble's stream (the members' home stream) and the member streams
  bool ok = cudaSetDevice(device) == cudaSuccess &&
            cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking) == cudaSuccess &&
            cudaEventCreateWithFlags(&e->fork, cudaEventDisableTiming) == cudaSuccess;
  for (int k = 0; ok && k < std::min(kEnsStreams, n); ++k) {
    cudaStream_t st = nullptr;
    cudaEvent_t ev = nullptr;
    ok = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) == cudaSuccess;
    if (ok) e->mstream.push_back(st);
    ok = ok && cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) == cudaSuccess;
    if (ok) e->join.push_back(ev);
  }
  if (!ok) {
    ens_destroy(e);
    g_create_error = "coral_ensemble_create: stream creation failed";
    return CORAL_ECUDA;
  }
  for (coral_handle* h : e->mem) {
    cudaStreamSynchronize(h->stream);
    cudaStreamDestroy(h->stream);
    h->stream = e->stream;
  }
  *out = e;
  return CORAL_OK;
}

void coral_ensemble_destroy(coral_ensemble* e) { ens_destroy(e); }

const char* coral_ensemble_last_error(const coral_ensemble* e) { return e ? e->err.c_str() : g_create_error.c_str(); }

int coral_ensemble_member(coral_ensemble* e, int i, coral_handle** member) {
  return ens_guarded(e, [&] {
    if (!member || i < 0 || i >= (int)e->mem.size()) throw CoralError(CORAL_EBADARG, "member index out of range");
    *member = e->mem[i];
  });
}

int coral_ensemble_march(coral_ensemble* e, double dt, int nsteps) {
  return ens_guarded(e, [&] { ens_march(e, dt, nsteps); });
}

int coral_ensemble_synchronize(coral_ensemble* e) {
  return ens_guarded(e, [&] {
    CK(cudaStreamSynchronize(e->stream));
    for (size_t i = 0; i < e->mem.size(); ++i) {
      unsigned int f = 0;
      CK(cudaMemcpy(&f, e->mem[i]->flags, sizeof(f), cudaMemcpyDeviceToHost));
      if (f & 1u) throw CoralError(CORAL_ENONFINITE, "non-finite value in the state of member " + std::to_string(i));
    }
  });
}

int coral_ensemble_query(coral_ensemble* e, int what, long long* value) {
  return ens_guarded(e, [&] {
    if (!value) throw CoralError(CORAL_EBADARG, "null pointer");
    switch (what) {
      case 0: *value = (long long)e->mem.size(); break;                 // members
      case 1: *value = e->launches; break;                              // kernels launched so far
      case 2: *value = e->batched ? 1 : 0; break;                       // substitutions batched
      case 3: *value = e->launches_per_step; break;                     // kernels per ensemble step
      default: throw CoralError(CORAL_EBADARG, "unknown ensemble query");
    }
  });
}

}  // extern "C"
