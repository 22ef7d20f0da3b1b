// CUDA kernels (sm_100a, FP64) of the plane-layer IMEX timestep.
//
// Layouts (first index slowest, C order), identical in memory to the
// reference's Fortran arrays:
//   state       field[kx][ky][t]          (Fortran field(T, NYAA, NX/2))
//   spectral    spec [kx][ky][n]          (Fortran spec(NZ, NYAA, NX/2))
//   physical    phys [y][x][z]            (Fortran phys(NZAA, NXAA, NYAA))
// Transform intermediates (this build's own choice):
//   Y1 / Q1     [var][y][kx][n]  complex  (after the y transform / before it)
//   Y2 / Q2     [var][y][x][n]   real     (after the x transform / before it)
// The x<->y exchange of the reference's slab decomposition
// (src/slabs.fftw3mpi/domain_decomposition.f90:152-183) is the change of
// layout between the y pass and the x pass, done in shared memory.
#include <algorithm>
#include <cstdio>

#include <string>

#include "../../include/coral_b200.h"
#include "device.hpp"
#include "host.hpp"

namespace coral {

namespace {

constexpr int kNB1 = 4;  // n lines per CTA, inverse / forward y pass
constexpr int kNB2 = 8;  // n lines per CTA, x passes (packed in pairs)
constexpr int kXB3 = 16; // x columns per CTA, inverse z pass (packed in pairs)
constexpr int kQC = 5;   // quadratic variables per FFT batch, forward z pass (one radix-9 / radix-8
                         // butterfly per thread at NZAA = 288)
constexpr int kPadY = 2;   // line stride of the y passes (kNB1 interleaved lines)
constexpr int kPadXY = 2;  // line stride N + 2 in the x / y passes, whose loads and stores
                           // walk 4 interleaved lines: 2 line + position hits 8 distinct
                           // 16-byte bank groups
constexpr int kThreads = 256;
// FFT plans of the time-step transforms (fft.cuh plan_of): the x passes and the
// fused z passes use the two-pass plans (576 = 24 x 24, 288 = 18 x 16); the y
// passes, whose first pass gathers its inputs (spectral build, strided
// coefficients), keep the three-pass plans with their shorter per-thread load
// chains (measured at 384^2 x 192)
constexpr int kPlanHot = 1;
constexpr int kPlanY = 0;
// x / y passes: threads per CTA for nl lines of a compiled length N, the most
// butterflies of any pass rounded up to whole warps (one butterfly per thread
// per pass); 256 for the run-time plans
__host__ __device__ constexpr int xy_threads(int N, int nl, int pv) {
  if (N == 0) return 256;
  const PlanR p = plan_of(N, pv);
  int m = 32;
  for (int i = 0; i < p.nst; ++i) m = (nl * N / p.r[i] > m) ? nl * N / p.r[i] : m;
  return (m + 31) / 32 * 32;
}
#define kThreadsX xy_threads(NF, kNB2 / 2, PV)
#define kThreadsY xy_threads(NF, 4, kPlanY)
// the pipelined forward y pass reads its first-pass inputs from shared memory:
// plan and threads of its own
constexpr int kPlanYF = 1;
#define kThreadsYF xy_threads(NF, 4, kPlanYF)
#define kMinBlocksYF (kPlanYF ? hot_min_blocks(kThreadsYF) : kMinBlocksY)
// CTAs per SM the kernels with two-pass plans are compiled for: registers
// capped at no fewer than 128 per thread
__host__ __device__ constexpr int hot_min_blocks(int nt) { return 65536 / (nt * 128) > 1 ? 65536 / (nt * 128) : 1; }
// CTAs per SM of the y passes (measured best at 384^2 x 192) and of the
// separate z passes of the transform API paths
constexpr int kMinBlocksY = 3;
constexpr int kMinBlocksZ = 4;
constexpr int kWPB = 8;  // warps (systems) per CTA in the per-system kernels

__device__ __forceinline__ double2 zero2() { return make_double2(0.0, 0.0); }

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}
// 16 bytes, or zeros when !valid (then gmem is not read)
__device__ __forceinline__ void cp_async16z(void* smem, const void* gmem, bool valid) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  const int n = valid ? 16 : 0;
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(sa), "l"(gmem), "r"(n) : "memory");
}


// 32-byte global store of two adjacent complex values (256-bit vector access;
// the address must be 32-byte aligned).  (The matching 32-byte load, tried for
// the inverse x pass's packed rows, was slower than two 16-byte loads.)
__device__ __forceinline__ void st32(double2* p, double2 a, double2 b) {
  asm volatile("st.global.v4.f64 [%0], {%1,%2,%3,%4};" ::"l"(p), "d"(a.x), "d"(a.y), "d"(b.x), "d"(b.y) : "memory");
}
__device__ __forceinline__ bool aligned32(const void* p) { return ((size_t)p & 31) == 0; }

__device__ __forceinline__ double2 ipow(double k, int e) {
  // (i k)^e by repeated multiplication, as Fortran's complex**integer
  double2 r = make_double2(1.0, 0.0);
  double2 z = make_double2(0.0, k);
  for (int q = 0; q < e; ++q) r = cmul(r, z);
  return r;
}

// ------------------------------------------------------------------------------
// inverse transform, pass 1: spectral build of the full variables + y c2c (e^{+i})
// (compute_full_variables_in_physical_space, marching.f90:436-503, then
//  c2r_transform steps 1-2 and the 0.5 of the x padding, transforms.f90:172-198)
// ------------------------------------------------------------------------------
template <int NF>
__global__ void __launch_bounds__(kThreadsY, kMinBlocksY) k_inv_y(Dims d, const FullVarDev* fv, StateSet st,
                                                     const double2* plain_spec, const double* kxv,
                                                     const double* kyv, double2* Y1, FftPlan py) {
  extern __shared__ double2 sm[];
  const int f = blockIdx.x, n0 = blockIdx.y * kNB1, kx = blockIdx.z;
  const int NYA = NF ? NF : d.NYA, LS = NYA + kPadY;
  double2* A = sm;
  double2* B = sm + kNB1 * LS;  // runtime plan only
  // the CTA's build tables in shared memory: per term and line the stencil's
  // state indices and values, the term's state base at this kx and (i kx)^dx,
  // so that the state loads of the first pass depend on no global load
  __shared__ int s_tt[kMaxFullTerms][kNB1][kTabW];
  __shared__ double s_tv[kMaxFullTerms][kNB1][kTabW];
  __shared__ const double2* s_base[kMaxFullTerms];
  __shared__ double2 s_kxf[kMaxFullTerms];
  __shared__ int s_kt[kMaxFullTerms], s_zero[kMaxFullTerms], s_dx[kMaxFullTerms], s_dy[kMaxFullTerms];
  __shared__ double s_dsca[kMaxFullTerms];
  const int nterms = plain_spec ? 0 : fv[f].nterms;
  for (int e = threadIdx.x; e < nterms * kNB1 * kTabW; e += blockDim.x) {
    const int t = e / (kNB1 * kTabW), r = e - t * kNB1 * kTabW, ln = r / kTabW, k = r - ln * kTabW;
    const FullTermDev& ft = fv[f].term[t];
    const int n = n0 + ln;
    s_tt[t][ln][k] = n < d.NZ ? ft.tab_t[n * kTabW + k] : -1;
    s_tv[t][ln][k] = n < d.NZ ? ft.tab_v[n * kTabW + k] : 0.0;
  }
  if (threadIdx.x < nterms) {
    const int t = threadIdx.x;
    const FullTermDev& ft = fv[f].term[t];
    s_zero[t] = ft.zero_kind;
    s_dx[t] = ft.dx;
    s_dy[t] = ft.dy;
    s_dsca[t] = ft.dsca;
    s_kt[t] = ft.zero_kind ? 0 : st.kT[ft.set];
    s_base[t] = ft.zero_kind ? nullptr : st.k[ft.set] + (size_t)kx * NYA * st.kT[ft.set];
    s_kxf[t] = ipow(kxv[kx], ft.dx);
  }
  __syncthreads();
  // the spectral build of (line ln = Chebyshev n0 + ln, ky index iy), produced
  // inside the first FFT pass
  auto ld = [&](int ln, int iy) -> double2 {
    const int n = n0 + ln;
    double2 c = zero2();
    if (n < d.NZ) {
      if (plain_spec) {
        c = plain_spec[((size_t)kx * NYA + iy) * d.NZ + n];
      } else {
        for (int t = 0; t < nterms; ++t) {
          if (s_zero[t]) {
            if (kx == 0 && iy == 0) {
              const FullTermDev& ft = fv[f].term[t];
              const double* zs = st.z[ft.set];
              double s = 0.0;
              for (int k = 0; k < kTabW; ++k) {
                int tt = ft.tab_t[n * kTabW + k];
                if (tt >= 0) s += ft.tab_v[n * kTabW + k] * zs[tt];
              }
              c.x += s * ft.dsca;
            }
          } else {
            const double2* sv = s_base[t] + (size_t)iy * s_kt[t];
            double2 s = zero2();
#pragma unroll
            for (int k = 0; k < kTabW; ++k) {
              const int tt = s_tt[t][ln][k];
              if (tt >= 0) {
                const double w = s_tv[t][ln][k];
                const double2 x = sv[tt];
                s.x += w * x.x;
                s.y += w * x.y;
              }
            }
            s = cscale(s, s_dsca[t]);
            if (s_dx[t] || s_dy[t]) s = cmul(cmul(s, s_kxf[t]), ipow(kyv[iy], s_dy[t]));
            c = cadd(c, s);
          }
        }
      }
    }
    return c;
  };
  const double2* R = fft_lines_ld<NF, true, kThreadsY, kNB1, true, kPlanY>(A, B, kNB1, LS, py, ld);
  for (int idx = threadIdx.x; idx < kNB1 * NYA; idx += blockDim.x) {
    const int ln = idx % kNB1, y = idx / kNB1, n = n0 + ln;
    if (n < d.NZ) {
      const double s = (n == 0) ? 1.0 : 0.5;  // (x2 on Chebyshev index 0) * (0.5 of the x padding)
      Y1[(((size_t)f * NYA + y) * d.NXH + kx) * d.NZ + n] = cscale(R[ln * LS + y], s);
    }
  }
}

// The same pass for full variables whose terms are mean variables followed by
// exactly one kxky variable (the u, v, w, T of the plane-layer recipes): the
// mean terms reach only the (0,0) mode and are summed in the prologue, in term
// order, so that a position's build is one unrolled stencil whose state loads
// do not wait on a loop over terms, and all of a thread's loads in the first
// pass can be in flight at once.  The same arithmetic in the same order as
// k_inv_y (bit for bit).
template <int NF>
__global__ void __launch_bounds__(kThreadsY, kMinBlocksY) k_inv_y1(Dims d, const FullVarDev* fv, StateSet st,
                                                      const double* kxv, const double* kyv, double2* Y1, FftPlan py) {
  extern __shared__ double2 sm[];
  const int f = blockIdx.x, n0 = blockIdx.y * kNB1, kx = blockIdx.z;
  const int NYA = NF ? NF : d.NYA, LS = NYA + kPadY;
  double2* A = sm;
  double2* B = sm + kNB1 * LS;  // runtime plan only
  __shared__ int s_tt[kNB1][kTabW];
  __shared__ double s_tv[kNB1][kTabW];
  __shared__ double2 s_zc[kNB1];  // per line, the mean terms' sum at (kx, ky) = (0, 0)
  const int tk = fv[f].nterms - 1;  // the kxky term is the last
  const FullTermDev& ft = fv[f].term[tk];
  for (int e = threadIdx.x; e < kNB1 * kTabW; e += blockDim.x) {
    const int ln = e / kTabW, k = e - ln * kTabW, n = n0 + ln;
    s_tt[ln][k] = n < d.NZ ? ft.tab_t[n * kTabW + k] : -1;
    s_tv[ln][k] = n < d.NZ ? ft.tab_v[n * kTabW + k] : 0.0;
  }
  if (threadIdx.x < kNB1) {
    const int ln = threadIdx.x, n = n0 + ln;
    double2 c = zero2();
    if (kx == 0 && n < d.NZ) {
      for (int t = 0; t < tk; ++t) {  // the mean terms, as k_inv_y's build at iy = 0
        const FullTermDev& fz = fv[f].term[t];
        const double* zs = st.z[fz.set];
        double s = 0.0;
        for (int k = 0; k < kTabW; ++k) {
          const int tt = fz.tab_t[n * kTabW + k];
          if (tt >= 0) s += fz.tab_v[n * kTabW + k] * zs[tt];
        }
        c.x += s * fz.dsca;
      }
    }
    s_zc[ln] = c;
  }
  const int kt = st.kT[ft.set], dx = ft.dx, dy = ft.dy;
  const double2* base = st.k[ft.set] + (size_t)kx * NYA * kt;
  const double dsca = ft.dsca;
  const double2 kxf = ipow(kxv[kx], dx);
  __syncthreads();
  auto ld = [&](int ln, int iy) -> double2 {
    const int n = n0 + ln;
    double2 c = zero2();
    if (n < d.NZ) {
      if (kx == 0 && iy == 0) c = s_zc[ln];
      const double2* sv = base + (size_t)iy * kt;
      double2 s = zero2();
#pragma unroll
      for (int k = 0; k < kTabW; ++k) {
        const int tt = s_tt[ln][k];
        if (tt >= 0) {
          const double w = s_tv[ln][k];
          const double2 x = sv[tt];
          s.x += w * x.x;
          s.y += w * x.y;
        }
      }
      s = cscale(s, dsca);
      if (dx || dy) s = cmul(cmul(s, kxf), ipow(kyv[iy], dy));
      c = cadd(c, s);
    }
    return c;
  };
  const double2* R = fft_lines_ld<NF, true, kThreadsY, kNB1, true, kPlanY>(A, B, kNB1, LS, py, ld);
  // two adjacent Chebyshev rows per thread: one 32-byte store
  for (int idx = threadIdx.x; idx < (kNB1 / 2) * NYA; idx += blockDim.x) {
    const int l0 = 2 * (idx % (kNB1 / 2)), y = idx / (kNB1 / 2), n = n0 + l0;
    // (x2 on Chebyshev index 0) * (0.5 of the x padding)
    const double2 v0 = cscale(R[l0 * LS + y], (n == 0) ? 1.0 : 0.5);
    const double2 v1 = cscale(R[(l0 + 1) * LS + y], 0.5);
    double2* dst = Y1 + (((size_t)f * NYA + y) * d.NXH + kx) * d.NZ + n;
    if (n + 1 < d.NZ && aligned32(dst)) {
      st32(dst, v0, v1);
    } else {
      if (n < d.NZ) dst[0] = v0;
      if (n + 1 < d.NZ) dst[1] = v1;
    }
  }
}

// ------------------------------------------------------------------------------
// inverse transform, pass 2: x c2r with zero padding NX/2 -> NXAA (transforms.f90:197-210)
// two real output lines per complex FFT
// ------------------------------------------------------------------------------
template <int NF, int PV>
__global__ void __launch_bounds__(kThreadsX, hot_min_blocks(kThreadsX)) k_inv_x(Dims d, const double2* Y1, double* Y2, FftPlan px,
                                                                               int y0) {
  extern __shared__ double2 sm[];
  const int f = blockIdx.x, n0 = blockIdx.y * kNB2, y = y0 + blockIdx.z;
  const int NXA = NF ? NF : d.NXA, NP = kNB2 / 2, LS = NXA + kPadXY;
  double2* A = sm;
  double2* B = sm + NP * LS;  // runtime plan only
  // position p of line m (Chebyshev pair na, na+1): the Hermitian extension of
  // both coefficient rows packed as a + i b, zero padding in between; produced
  // inside the first FFT pass
  const double2* src0 = Y1 + ((size_t)f * d.NYA + y) * d.NXH * d.NZ;
  auto ld = [&](int m, int p) -> double2 {
    const int na = n0 + 2 * m;
    const bool lo = p < d.NXH, hi = p > NXA - d.NXH;  // kx = p, or kx = NXA - p (conjugate)
    if (!lo && !hi) return zero2();
    const int kx = lo ? p : NXA - p;
    const double2* src = src0 + (size_t)kx * d.NZ;
    const double2 a = (na < d.NZ) ? src[na] : zero2();
    const double2 b = (na + 1 < d.NZ) ? src[na + 1] : zero2();
    if (p == 0) return make_double2(a.x, b.x);  // c2r reads only the real part of the DC term
    return lo ? make_double2(a.x - b.y, a.y + b.x)    // a + i b
              : make_double2(a.x + b.y, b.x - a.y);   // conj(a) + i conj(b)
  };
  const double2* R = fft_lines_ld<NF, true, kThreadsX, kNB2 / 2, true, PV>(A, B, NP, LS, px, ld);
  for (int idx = threadIdx.x; idx < NP * NXA; idx += blockDim.x) {
    const int m = idx % NP, x = idx / NP, na = n0 + 2 * m;
    double2 z = R[m * LS + x];
    double* dst = Y2 + (((size_t)f * d.NYA + y) * NXA + x) * d.NZ;
    if (na + 1 < d.NZ && (d.NZ & 1) == 0) {
      *reinterpret_cast<double2*>(dst + na) = z;  // na and NZ even: one 16-byte store
    } else {
      if (na < d.NZ) dst[na] = z.x;
      if (na + 1 < d.NZ) dst[na + 1] = z.y;
    }
  }
}

// The same pass for compiled lengths with the two-pass plan, as a persistent
// kernel: each CTA walks the tiles (full variable, block of kNB2 Chebyshev rows,
// y) with a stride of the grid size; the next tile's input rows (kx < NX/2,
// kNB2 coefficients each) are copied into a staging buffer with cp.async while
// the current tile's second FFT pass and stores run (the first pass reads the
// staging buffer and frees it).  Staging rows are kNB2 + 1 16-byte words apart,
// so that the first pass's reads (4 lines x 2 positions a quarter warp) fall in
// distinct bank groups; the second pass reads its twiddles from the
// conflict-free table of build_tw_pass2.  Shared memory (line buffer, staging,
// table) admits 3 CTAs per SM at NXAA = 576: registers are sized for 3.
constexpr int kStgX = kNB2 + 1;
#define kThreadsXP xy_threads(NF, kNB2 / 2, 1)
template <int NF>
__global__ void __launch_bounds__(kThreadsXP, 3) k_inv_x_pipe(Dims d, int nf, const double2* Y1,
                                                                                      double* Y2, FftPlan px) {
  constexpr int NT = kThreadsXP, NXA = NF, NP = kNB2 / 2;
  constexpr PlanR P = plan_of(NF, 1);
  constexpr int kTw2 = tw_pass2_len<NF, 1>();
  static_assert(kTw2 > 0, "two-pass plan");
  extern __shared__ double2 sm[];
  __shared__ double2 s_tw[kTw2];
  const int LS = NXA + kPadXY;
  double2* A = sm;               // NP lines, stride LS
  double2* stg = A + NP * LS;    // staged input [kx][kStgX]
  const int NXH = d.NXH, NZ = d.NZ;
  const int nnb = (NZ + kNB2 - 1) / kNB2;
  const int ntiles = nf * nnb * d.NYA;
  build_tw_pass2<NF, 1>(s_tw, px.tw);  // read after the loop's first barrier
  auto issue = [&](int tile) {
    if (tile < ntiles) {
      const int f = tile % nf, r = tile / nf, nb = r % nnb, y = r / nnb, n0 = nb * kNB2;
      const double2* src = Y1 + ((size_t)f * d.NYA + y) * NXH * NZ + n0;
      for (int e = threadIdx.x; e < NXH * kNB2; e += NT) {
        const int kx = e / kNB2, ln = e - kx * kNB2;
        const bool ok = n0 + ln < NZ;
        cp_async16z(stg + kx * kStgX + ln, ok ? src + (size_t)kx * NZ + ln : Y1, ok);
      }
    }
    cp_async_commit();
  };
  issue(blockIdx.x);
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int f = tile % nf, r = tile / nf, nb = r % nnb, y = r / nnb, n0 = nb * kNB2;
    cp_async_wait<0>();
    __syncthreads();
    // position p of line m (Chebyshev pair 2m, 2m+1 of the block): as in k_inv_x
    auto ld = [&](int m, int p) -> double2 {
      const bool lo = p < NXH, hi = p > NXA - NXH;
      if (!lo && !hi) return zero2();
      const int kx = lo ? p : NXA - p;
      const double2 a = stg[kx * kStgX + 2 * m], b = stg[kx * kStgX + 2 * m + 1];
      if (p == 0) return make_double2(a.x, b.x);
      return lo ? make_double2(a.x - b.y, a.y + b.x) : make_double2(a.x + b.y, b.x - a.y);
    };
    fft_pass_first<NF, P.r[0], true, NT, NP, true>(A, NP, LS, ld);  // ends with a barrier
    issue(tile + gridDim.x);
    fft_passes<NF, 1, P.r[0], true, NT, NP, 1, true>(A, NP, LS, s_tw);
    double* dst0 = Y2 + ((size_t)f * d.NYA + y) * NXA * NZ;
    for (int idx = threadIdx.x; idx < NP * NXA; idx += NT) {
      const int m = idx % NP, x = idx / NP, na = n0 + 2 * m;
      const double2 z = A[m * LS + x];
      double* dst = dst0 + (size_t)x * NZ + na;
      if (na + 1 < NZ && (NZ & 1) == 0) {
        *reinterpret_cast<double2*>(dst) = z;  // na and NZ even: 16-byte aligned
      } else {
        if (na < NZ) dst[0] = z.x;
        if (na + 1 < NZ) dst[1] = z.y;
      }
    }
    __syncthreads();  // A is rewritten by the next tile's first pass
  }
  cp_async_wait<0>();
}

__device__ __forceinline__ void atomic_max_nonneg(unsigned long long* addr, double v) {
  atomicMax(addr, (unsigned long long)__double_as_longlong(v));
}

// ------------------------------------------------------------------------------
// inverse transform, pass 3: z REDFT01 with zero padding NZ -> NZAA (transforms.f90:216-223)
// via an NZAA-point complex FFT (two columns per FFT); also the CFL maxima of
// compute_cfl_based_timestep (marching.f90:219-238) for the first three full variables
// ------------------------------------------------------------------------------
template <int NF>
__global__ void __launch_bounds__(kThreads, kMinBlocksZ) k_inv_z(Dims d, const double* Y2, double* phys, FftPlan pz,
                                                     const double2* dct_tw, const double* wz,
                                                     unsigned long long* cfl_bits) {
  extern __shared__ double2 sm[];
  __shared__ double red[kThreads / 32];
  const int f = blockIdx.x, x0 = blockIdx.y * kXB3, y = blockIdx.z;
  const int N = NF ? NF : d.NZA, NP = kXB3 / 2;
  double2* A = sm;
  double2* B = sm + NP * N;
  for (int idx = threadIdx.x; idx < NP * N; idx += blockDim.x) {
    const int m = idx / N, n = idx - m * N;
    const int xa = x0 + 2 * m, xb = xa + 1;
    const double* sa = Y2 + (((size_t)f * d.NYA + y) * d.NXA + xa) * d.NZ;
    const double* sb = sa + d.NZ;
    double a0 = 0, a1 = 0, b0 = 0, b1 = 0;  // X_n, X_{N-n}
    if (xa < d.NXA) {
      if (n < d.NZ) a0 = sa[n];
      if (n > 0 && N - n < d.NZ) a1 = sa[N - n];
    }
    if (xb < d.NXA) {
      if (n < d.NZ) b0 = sb[n];
      if (n > 0 && N - n < d.NZ) b1 = sb[N - n];
    }
    const double2 w = cconj(dct_tw[n]);  // exp(+i pi n / 2N)
    double2 va = cmul(w, make_double2(a0, -a1));
    double2 vb = cmul(w, make_double2(b0, -b1));
    A[m * N + n] = make_double2(va.x - vb.y, va.y + vb.x);  // va + i vb
  }
  __syncthreads();
  const double2* R = fft_lines_n<NF, true, kThreads, kXB3 / 2>(A, B, NP, N, pz);
  double mx = 0.0;
  const int which = (f < 3) ? f : -1;
  for (int idx = threadIdx.x; idx < NP * N; idx += blockDim.x) {
    const int m = idx / N, k = idx - m * N;
    const int xa = x0 + 2 * m, xb = xa + 1;
    const int zi = (k & 1) ? (N - 1 - (k >> 1)) : (k >> 1);
    const double2 z = R[m * N + zi];
    double* dst = phys + (((size_t)f * d.NYA + y) * d.NXA + xa) * N;
    if (xa < d.NXA) dst[k] = z.x;
    if (xb < d.NXA) dst[N + k] = z.y;
    if (which >= 0) {
      double s = (which == 2) ? 1.0 / wz[k] : 1.0;
      if (xa < d.NXA) mx = fmax(mx, fabs(z.x) * s);
      if (xb < d.NXA) mx = fmax(mx, fabs(z.y) * s);
    }
  }
  if (cfl_bits && which >= 0) {
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = mx;
    __syncthreads();
    if (threadIdx.x == 0) {
      double m2 = 0.0;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) m2 = fmax(m2, red[w]);
      atomic_max_nonneg(cfl_bits + which, m2);
    }
  }
}

// ------------------------------------------------------------------------------
// forward transform, pass 1: pointwise products (marching.f90:279-291) + z REDFT10
// truncated to NZ (transforms.f90:243-249), for all quadratic variables of one
// pair of x columns; also partial volume averages for KE (output.f90:84-102)
// ------------------------------------------------------------------------------
template <int NF>
__global__ void __launch_bounds__(kThreads, kMinBlocksZ) k_fwd_z(Dims d, int nf, QuadDesc q, const double* phys, double* Q2,
                                                     FftPlan pz, const double2* dct_tw, const double* wz,
                                                     double* ke_partial) {
  extern __shared__ double2 sm[];
  __shared__ double red[3][kThreads / 32];
  const int x0 = blockIdx.x * 2, y = blockIdx.y;
  const int N = NF ? NF : d.NZA, nq = q.nq, nb = min(nq, kQC);
  double* P = reinterpret_cast<double*>(sm);  // [nf][2][N], z in Makhoul order
  double2* A = sm + nf * N;                    // nb lines
  double2* B = A + nb * N;                     // runtime plan only
  for (int idx = threadIdx.x; idx < nf * 2 * N; idx += blockDim.x) {
    const int fv = idx / (2 * N), r = idx - fv * 2 * N;
    const int c = r / N, z = r - c * N;
    const int m = (z & 1) ? (N - 1 - (z >> 1)) : (z >> 1);  // Makhoul position of z
    const int xc = x0 + c;
    P[idx - z + m] = (xc < d.NXA) ? phys[(((size_t)fv * d.NYA + y) * d.NXA + xc) * N + z] : 0.0;
  }
  __syncthreads();
  double ke[3] = {0.0, 0.0, 0.0};
  for (int q0 = 0; q0 < nq; q0 += kQC) {  // batches of kQC quadratic variables
    const int nc = min(kQC, nq - q0);
    for (int idx = threadIdx.x; idx < nc * N; idx += blockDim.x) {
      const int qi = idx / N, m = idx - qi * N, qg = q0 + qi;
      const int z = (m < N / 2) ? 2 * m : 2 * (N - 1 - m) + 1;  // Makhoul reordering
      const int v1 = q.v1[qg], v2 = q.v2[qg];
      double pa, pb;
      if (v1 < 0) { pa = P[(v2 * 2) * N + m]; pb = P[(v2 * 2 + 1) * N + m]; }
      else if (v2 < 0) { pa = P[(v1 * 2) * N + m]; pb = P[(v1 * 2 + 1) * N + m]; }
      else {
        pa = P[(v1 * 2) * N + m] * P[(v2 * 2) * N + m];
        pb = P[(v1 * 2 + 1) * N + m] * P[(v2 * 2 + 1) * N + m];
      }
      if (ke_partial) {
        for (int j = 0; j < 3; ++j)
          if (q.ke_q[j] == qg) ke[j] += wz[z] * (pa + ((x0 + 1 < d.NXA) ? pb : 0.0));
      }
      if (q.tau) {  // learned subgrid part of this quadratic variable
        const double* tq = q.tau + (((size_t)qg * d.NYA + y) * d.NXA + x0) * N + z;
        pa += tq[0];
        if (x0 + 1 < d.NXA) pb += tq[N];
      }
      A[qi * N + m] = make_double2(pa, pb);
    }
    __syncthreads();
    const double2* R = fft_lines_n<NF, false, kThreads, kQC>(A, B, nc, N, pz);
    for (int idx = threadIdx.x; idx < nc * d.NZ; idx += blockDim.x) {
      const int qi = idx / d.NZ, n = idx - qi * d.NZ;
      const double2 Z = R[qi * N + n];
      const double2 Zc = cconj(R[qi * N + ((N - n) % N)]);
      const double2 va = make_double2(0.5 * (Z.x + Zc.x), 0.5 * (Z.y + Zc.y));
      const double2 dd = csub(Z, Zc);
      const double2 vb = make_double2(0.5 * dd.y, -0.5 * dd.x);  // (Z - Zc) / 2i
      const double2 w = dct_tw[n];                                // exp(-i pi n / 2N)
      const double xa = 2.0 * (w.x * va.x - w.y * va.y);
      const double xb = 2.0 * (w.x * vb.x - w.y * vb.y);
      double* dst = Q2 + (((size_t)(q0 + qi) * d.NYA + y) * d.NXA + x0) * d.NZ;
      dst[n] = xa;
      if (x0 + 1 < d.NXA) dst[d.NZ + n] = xb;
    }
    __syncthreads();  // A is refilled by the next batch
  }
  if (ke_partial) {
    for (int j = 0; j < 3; ++j) {
      double v = ke[j];
      for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      if ((threadIdx.x & 31) == 0) red[j][threadIdx.x >> 5] = v;
    }
    __syncthreads();
    if (threadIdx.x < 3) {
      double s = 0.0;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[threadIdx.x][w];
      ke_partial[((size_t)blockIdx.y * gridDim.x + blockIdx.x) * 3 + threadIdx.x] = s;
    }
  }
}

// ------------------------------------------------------------------------------
// z passes of one stage fused: z REDFT01 of the full variables (transforms.f90:
// 216-223), the CFL maxima (marching.f90:219-238), the pointwise products
// (marching.f90:279-291), the KE partial averages (output.f90:84-102) and the z
// REDFT10 of the quadratic variables (transforms.f90:243-249), for one pair of
// x columns; the physical fields never leave shared memory.  The inverse
// transform leaves the physical values in Makhoul order (position m holds
// z = 2m, or 2(N-1-m)+1 for m >= N/2), which is the order the forward transform
// takes, so the products are formed position by position.
// ------------------------------------------------------------------------------

// Threads of the fused z kernel for nl lines of a compiled length N: enough for
// one butterfly per thread in the radix >= 8 passes and two in the radix-2/4
// passes (N = 288, 8 lines, plan 18 x 16: 160 threads).
__host__ __device__ constexpr int z_threads(int N, int nl) {
  if (N == 0) return 256;
  const PlanR p = plan_of(N, kPlanHot);
  int m = 32;
  for (int i = 0; i < p.nst; ++i) {
    const int b = nl * N / p.r[i], per = (p.r[i] <= 4) ? (b + 1) / 2 : b;
    m = per > m ? per : m;
  }
  return (m + 31) / 32 * 32;
}
constexpr int kZPairs = 2;               // x-column pairs per CTA
constexpr int kZLines = 4 * kZPairs;     // lines per inverse FFT batch (4 full variables x 2 pairs)
// lines per forward FFT batch ((quadratic variable, pair) lines), the kernel's
// FB: 9 (two batches for 9 quadratic variables; 2 CTAs per SM at NZAA = 288) or
// 6 (three batches; shared memory and registers for 3 CTAs per SM)
constexpr int kZFwd = 9;
__host__ __device__ constexpr int z_threads_fused(int N, int fb) {
  return z_threads(N, kZLines) > z_threads(N, fb) ? z_threads(N, kZLines) : z_threads(N, fb);
}
__host__ __device__ constexpr int z_min_blocks(int N, int fb) {
  return fb < kZFwd ? 3 : hot_min_blocks(z_threads_fused(N, fb));
}
#define kThreadsZF z_threads_fused(NF, FB)

template <int NF, int FB>
__global__ void __launch_bounds__(kThreadsZF, z_min_blocks(NF, FB)) k_z_fused(Dims d, int nf, QuadDesc q, const double* Y2,
                                                                       double* Q2, FftPlan pz, const double2* dct_tw,
                                                                       const double* wz, const double* wzinv,
                                                                       unsigned long long* cfl_bits, double* ke_partial,
                                                                       int y0) {
  constexpr int NT = kThreadsZF;
  extern __shared__ double2 sm[];
  __shared__ double red[3][(NT + 31) / 32];
  __shared__ int qv[2][kMaxQuad];
  const int x0 = blockIdx.x * 2 * kZPairs, y = y0 + blockIdx.y;
  const size_t cta = (size_t)y * gridDim.x + blockIdx.x;  // row of the KE and timeseries partial sums
  // compiled lengths: NZAA = 3 NZ / 2 (the launcher checks it)
  const int N = NF ? NF : d.NZA, NZ = NF ? 2 * NF / 3 : d.NZ;
  const int nq = q.nq;
  const size_t vstride = (size_t)d.NYA * d.NXA * NZ;  // between variables of Y2 / Q2
  const size_t col0 = ((size_t)y * d.NXA + x0) * NZ;  // column x0 of variable 0
  if (threadIdx.x < kMaxQuad) {
    qv[0][threadIdx.x] = q.v1[threadIdx.x];
    qv[1][threadIdx.x] = q.v2[threadIdx.x];
  }
  // compiled lengths: the FFT and DCT twiddles in shared memory; with a
  // two-pass plan the FFT twiddles as the bank-conflict-free pass-2 table
  constexpr int kTw2 = NF ? tw_pass2_len<NF, kPlanHot>() : 0;
  constexpr bool kTwl = kTw2 > 0;
  __shared__ double2 s_tw[kTwl ? kTw2 : (NF ? NF : 1)], s_dtw[NF ? NF : 1];
  FftPlan pzl = pz;
  const double2* dtw = dct_tw;
  if constexpr (NF != 0) {
    if constexpr (kTwl) {
      build_tw_pass2<NF, kPlanHot>(s_tw, pz.tw);
    } else {
      for (int i = threadIdx.x; i < NF; i += blockDim.x) s_tw[i] = pz.tw[i];
    }
    for (int i = threadIdx.x; i < NF; i += blockDim.x) s_dtw[i] = dct_tw[i];
    pzl.tw = s_tw;
    dtw = s_dtw;
  }
  // line l of a batch: variable l / kZPairs, column pair l % kZPairs (columns
  // x0 + 2p (re) and x0 + 2p + 1 (im))
  auto col_ok = [&](int c) { return x0 + c < d.NXA; };
  double2* Fv = sm;                   // nf * kZPairs lines of the full variables
  double2* A = Fv + nf * kZPairs * N; // FB lines of quadratic variables
  double2* B = A + FB * N;            // runtime plan only (max(kZLines, FB) lines)
  // ---- inverse: X_n and X_{N-n} of both columns, twiddled, packed as va + i vb,
  //      produced inside the first FFT pass ----
  __syncthreads();  // qv
  for (int l0 = 0; l0 < nf * kZPairs; l0 += kZLines) {
    const int nl = min(kZLines, nf * kZPairs - l0);
    auto ld = [&](int line, int n) -> double2 {
      const int lg = l0 + line, f = lg / kZPairs, pr = lg - f * kZPairs;
      const bool ha = col_ok(2 * pr), hb = col_ok(2 * pr + 1);
      const double* sa = Y2 + f * vstride + col0 + (size_t)(2 * pr) * NZ;
      const double* sb = sa + NZ;
      const bool lo = n < NZ, hi = n > 0 && N - n < NZ;
      const double a0 = (lo && ha) ? sa[n] : 0.0, a1 = (hi && ha) ? sa[N - n] : 0.0;
      const double b0 = (lo && hb) ? sb[n] : 0.0, b1 = (hi && hb) ? sb[N - n] : 0.0;
      const double2 w = cconj(dtw[n]);  // exp(+i pi n / 2N)
      const double2 va = cmul(w, make_double2(a0, -a1));
      const double2 vb = cmul(w, make_double2(b0, -b1));
      return make_double2(va.x - vb.y, va.y + vb.x);
    };
    const double2* R = fft_lines_ld<NF, true, NT, kZLines, false, kPlanHot, kTwl>(Fv + l0 * N, B, nl, N, pzl, ld);
    if (R != Fv + l0 * N) {  // runtime plan with the result in the scratch lines
      for (int idx = threadIdx.x; idx < nl * N; idx += blockDim.x) Fv[l0 * N + idx] = R[idx];
      __syncthreads();
    }
  }
  // full variables with given physical values replace their transforms
  if (q.st_n > 0) {
    for (int k = 0; k < q.st_n; ++k) {
      const double* src = q.st_src[k];
      const int f = q.st_var[k], prof = q.st_prof[k];
      for (int idx = threadIdx.x; idx < kZPairs * N; idx += blockDim.x) {
        const int pr = idx / N, m = idx - pr * N;
        const int z = (m < N / 2) ? 2 * m : 2 * (N - 1 - m) + 1;
        double a = 0.0, b = 0.0;
        if (prof) {
          a = b = src[z];
        } else {
          const size_t at = ((size_t)y * d.NXA + x0 + 2 * pr) * N + z;
          if (col_ok(2 * pr)) a = src[at];
          if (col_ok(2 * pr + 1)) b = src[at + N];
        }
        Fv[(f * kZPairs + pr) * N + m] = make_double2(a, b);
      }
    }
    __syncthreads();
  }
  // ---- CFL maxima of |u|, |v|, |w| / wz and the KE sums (z-weighted products
  //      of the quadratic variables uu, vv, ww) over all columns, from the
  //      physical values (Makhoul order: position m is grid point z) ----
  if (cfl_bits || ke_partial) {
    const int ncf = cfl_bits ? min(nf, 3) : 0;
    double mx[3] = {0.0, 0.0, 0.0}, ke[3] = {0.0, 0.0, 0.0};
    for (int idx = threadIdx.x; idx < kZPairs * N; idx += blockDim.x) {
      const int pr = idx / N, m = idx - pr * N;
      const bool oka = col_ok(2 * pr), okb = col_ok(2 * pr + 1);
      const int z = (m < N / 2) ? 2 * m : 2 * (N - 1 - m) + 1;
#pragma unroll
      for (int j = 0; j < 3; ++j)
        if (j < ncf) {
          const double2 v = Fv[(j * kZPairs + pr) * N + m];
          const double s = (j == 2) ? wzinv[z] : 1.0;
          double a = oka ? fabs(v.x) * s : 0.0;
          if (okb) a = fmax(a, fabs(v.y) * s);
          mx[j] = fmax(mx[j], a);
        }
      if (ke_partial) {
        const double w = wz[z];
#pragma unroll
        for (int j = 0; j < 3; ++j) {
          const int qg = q.ke_q[j];
          if (qg < 0) continue;
          const int v1 = qv[0][qg], v2 = qv[1][qg];
          double pa, pb;
          if (v1 < 0 || v2 < 0) {
            const double2 f1 = Fv[((v1 < 0 ? v2 : v1) * kZPairs + pr) * N + m];
            pa = f1.x;
            pb = f1.y;
          } else {
            const double2 f1 = Fv[(v1 * kZPairs + pr) * N + m], f2 = Fv[(v2 * kZPairs + pr) * N + m];
            pa = f1.x * f2.x;
            pb = f1.y * f2.y;
          }
          ke[j] += w * ((oka ? pa : 0.0) + (okb ? pb : 0.0));
        }
      }
    }
    if (cfl_bits) {
      for (int j = 0; j < 3; ++j) {
        double v = mx[j];
        for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
        if ((threadIdx.x & 31) == 0) red[j][threadIdx.x >> 5] = v;
      }
      __syncthreads();
      if (threadIdx.x < ncf) {
        double m2 = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) m2 = fmax(m2, red[threadIdx.x][w]);
        atomic_max_nonneg(cfl_bits + threadIdx.x, m2);
      }
      __syncthreads();
    }
    if (ke_partial) {
      for (int j = 0; j < 3; ++j) {
        double v = ke[j];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if ((threadIdx.x & 31) == 0) red[j][threadIdx.x >> 5] = v;
      }
      __syncthreads();
      if (threadIdx.x < 3) {
        double s = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[threadIdx.x][w];
        ke_partial[cta * 3 + threadIdx.x] = s;
      }
      __syncthreads();
    }
    // timeseries objects, one at a time (one accumulator register)
    if (ke_partial && q.ts_partial) {
      for (int o = 0; o < q.ts_n; ++o) {
        const int src = q.ts_src[o], zsel = q.ts_z[o];
        const int fa = src >= 0 ? src : qv[0][-1 - src], fb = src >= 0 ? -1 : qv[1][-1 - src];
        double acc = 0.0;
        for (int idx = threadIdx.x; idx < kZPairs * N; idx += blockDim.x) {
          const int pr = idx / N, m = idx - pr * N;
          const int z = (m < N / 2) ? 2 * m : 2 * (N - 1 - m) + 1;
          if (zsel >= 0 && z != zsel) continue;
          double pa, pb;
          if (fa < 0 || fb < 0) {
            const double2 f1 = Fv[((fa < 0 ? fb : fa) * kZPairs + pr) * N + m];
            pa = f1.x;
            pb = f1.y;
          } else {
            const double2 f1 = Fv[(fa * kZPairs + pr) * N + m], f2 = Fv[(fb * kZPairs + pr) * N + m];
            pa = f1.x * f2.x;
            pb = f1.y * f2.y;
          }
          const double w = zsel >= 0 ? 1.0 : wz[z];
          acc += w * ((col_ok(2 * pr) ? pa : 0.0) + (col_ok(2 * pr + 1) ? pb : 0.0));
        }
        for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
        if ((threadIdx.x & 31) == 0) red[0][threadIdx.x >> 5] = acc;
        __syncthreads();
        if (threadIdx.x == 0) {
          double s = 0.0;
          for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[0][w];
          q.ts_partial[cta * kMaxTs + o] = s;
        }
        __syncthreads();
      }
    }
  }
  // ---- products and forward transforms, FB (quadratic variable, pair) lines a batch ----
  for (int l0 = 0; l0 < nq * kZPairs; l0 += FB) {
    const int nc = min(FB, nq * kZPairs - l0);
    // products formed inside the first FFT pass
    auto ld = [&](int line, int m) -> double2 {
      const int lg = l0 + line, qg = lg / kZPairs, pr = lg - qg * kZPairs;
      const int v1 = qv[0][qg], v2 = qv[1][qg];
      double pa, pb;
      if (v1 < 0 || v2 < 0) {
        const double2 f1 = Fv[((v1 < 0 ? v2 : v1) * kZPairs + pr) * N + m];
        pa = f1.x;
        pb = f1.y;
      } else {
        const double2 f1 = Fv[(v1 * kZPairs + pr) * N + m], f2 = Fv[(v2 * kZPairs + pr) * N + m];
        pa = f1.x * f2.x;
        pb = f1.y * f2.y;
      }
      return make_double2(pa, pb);
    };
    const double2* R = fft_lines_ld<NF, false, NT, FB, false, kPlanHot, kTwl>(A, B, nc, N, pzl, ld);
    // coefficient n of the two packed columns from Z = R[n] and conj(R[N - n]);
    // coefficients n and N - n share those two loads: items n = 0 .. N/2 write
    // n (< NZ) and, for 0 < n < N/2, N - n when it is < NZ
    const int NH = N / 2 + 1;
    for (int idx = threadIdx.x; idx < nc * NH; idx += blockDim.x) {
      const int li = idx / NH, n = idx - li * NH;
      const int lg = l0 + li, qg = lg / kZPairs, pr = lg - qg * kZPairs;
      const int n2 = (n == 0) ? 0 : N - n;
      const double2 Z = R[li * N + n], W = R[li * N + n2];
      double* dst = Q2 + qg * vstride + col0 + (size_t)(2 * pr) * NZ;
      const bool oa = col_ok(2 * pr), ob = col_ok(2 * pr + 1);
      auto out = [&](int k, double2 P, double2 Pm) {  // coefficient k from R[k] = P, R[N - k] = Pm
        const double2 Pc = cconj(Pm);
        const double2 va = make_double2(0.5 * (P.x + Pc.x), 0.5 * (P.y + Pc.y));
        const double2 dd = csub(P, Pc);
        const double2 vb = make_double2(0.5 * dd.y, -0.5 * dd.x);  // (P - Pc) / 2i
        const double2 w = dtw[k];                                   // exp(-i pi k / 2N)
        if (oa) dst[k] = 2.0 * (w.x * va.x - w.y * va.y);
        if (ob) dst[NZ + k] = 2.0 * (w.x * vb.x - w.y * vb.y);
      };
      if (n < NZ) out(n, Z, W);
      if (n > 0 && n2 != n && n2 < NZ) out(n2, W, Z);
    }
    __syncthreads();  // A is refilled by the next batch
  }
}

// ------------------------------------------------------------------------------
// forward transform, pass 2: x r2c, keep kx < NX/2 (transforms.f90:255-267)
// ------------------------------------------------------------------------------
template <int NF, int PV>
__global__ void __launch_bounds__(kThreadsX, hot_min_blocks(kThreadsX)) k_fwd_x(Dims d, const double* Q2, double2* Q1, FftPlan px,
                                                                               int y0) {
  extern __shared__ double2 sm[];
  const int qi = blockIdx.x, n0 = blockIdx.y * kNB2, y = y0 + blockIdx.z;
  const int NXA = NF ? NF : d.NXA, NP = kNB2 / 2, LS = NXA + kPadXY;
  double2* A = sm;
  double2* B = sm + NP * LS;  // runtime plan only
  // rows na, na+1 of column x packed as one complex value, produced inside the
  // first FFT pass
  const double* src0 = Q2 + ((size_t)qi * d.NYA + y) * NXA * d.NZ;
  auto ld = [&](int m, int x) -> double2 {
    const int na = n0 + 2 * m;
    const double* src = src0 + (size_t)x * d.NZ;
    if (na + 1 < d.NZ && (d.NZ & 1) == 0) return *reinterpret_cast<const double2*>(src + na);  // 16-byte aligned
    return make_double2(na < d.NZ ? src[na] : 0.0, na + 1 < d.NZ ? src[na + 1] : 0.0);
  };
  const double2* R = fft_lines_ld<NF, false, kThreadsX, kNB2 / 2, true, PV>(A, B, NP, LS, px, ld);
  for (int idx = threadIdx.x; idx < NP * d.NXH; idx += blockDim.x) {
    const int m = idx % NP, kx = idx / NP, na = n0 + 2 * m;
    const double2 Z = R[m * LS + kx];
    const double2 Zc = cconj(R[m * LS + ((NXA - kx) % NXA)]);
    const double2 a = make_double2(0.5 * (Z.x + Zc.x), 0.5 * (Z.y + Zc.y));
    const double2 dd = csub(Z, Zc);
    const double2 b = make_double2(0.5 * dd.y, -0.5 * dd.x);
    double2* dst = Q1 + (((size_t)qi * d.NYA + y) * d.NXH + kx) * d.NZ;
    if (na + 1 < d.NZ && aligned32(dst + na)) {
      st32(dst + na, a, b);  // rows na, na + 1: one 32-byte store
    } else {
      if (na < d.NZ) dst[na] = a;
      if (na + 1 < d.NZ) dst[na + 1] = b;
    }
  }
}

// ------------------------------------------------------------------------------
// forward transform, pass 3: y c2c (e^{-i}), x0.5 on Chebyshev index 0 and the
// 1/(NXAA NYAA NZAA) normalisation (transforms.f90:280-296)
// ------------------------------------------------------------------------------
template <int NF>
__global__ void __launch_bounds__(kThreadsY, kMinBlocksY) k_fwd_y(Dims d, const double2* Q1, double2* qspec, double scale,
                                                     FftPlan py) {
  extern __shared__ double2 sm[];
  const int qi = blockIdx.x, n0 = blockIdx.y * kNB1, kx = blockIdx.z;
  const int NYA = NF ? NF : d.NYA, LS = NYA + kPadY;
  double2* A = sm;
  double2* B = sm + kNB1 * LS;  // runtime plan only
  // produced inside the first FFT pass
  auto ld = [&](int ln, int y) -> double2 {
    const int n = n0 + ln;
    double2 v = zero2();
    if (n < d.NZ) {
      v = Q1[(((size_t)qi * NYA + y) * d.NXH + kx) * d.NZ + n];
      if (n == 0) v = cscale(v, 0.5);
    }
    return v;
  };
  const double2* R = fft_lines_ld<NF, false, kThreadsY, kNB1, true, kPlanY>(A, B, kNB1, LS, py, ld);
  for (int idx = threadIdx.x; idx < kNB1 * NYA; idx += blockDim.x) {
    const int ln = idx % kNB1, ky = idx / kNB1, n = n0 + ln;
    if (n < d.NZ) qspec[(((size_t)qi * d.NXH + kx) * NYA + ky) * d.NZ + n] = cscale(R[ln * LS + ky], scale);
  }
}

// The same pass for compiled lengths as a persistent kernel: each CTA walks the
// tiles (quadratic variable, block of kNB1 Chebyshev rows, kx) with a stride of
// the grid size; the next tile's input is copied into a staging buffer with
// cp.async while the current tile's later FFT passes and stores run (the first
// pass reads the staging buffer and frees it).
template <int NF>
__global__ void __launch_bounds__(kThreadsYF, kMinBlocksYF) k_fwd_y_pipe(Dims d, int nq, const double2* Q1,
                                                                        double2* qspec, double scale, FftPlan py) {
  extern __shared__ double2 sm[];
  constexpr int NYA = NF;
  constexpr PlanR P = plan_of(NF, kPlanYF);
  const int LS = NYA + kPadY;
  double2* A = sm;                 // kNB1 lines, stride LS
  double2* stg = A + kNB1 * LS;    // staged input [y][kNB1]
  const int nnb = (d.NZ + kNB1 - 1) / kNB1;
  const int ntiles = nq * nnb * d.NXH;
  const size_t ystride = (size_t)d.NXH * d.NZ;
  auto issue = [&](int tile) {
    if (tile < ntiles) {
      const int qi = tile % nq, r = tile / nq, nb = r % nnb, kx = r / nnb, n0 = nb * kNB1;
      const double2* src = Q1 + ((size_t)qi * NYA * d.NXH + kx) * d.NZ + n0;
      for (int e = threadIdx.x; e < NYA * kNB1; e += blockDim.x) {
        const int y = e / kNB1, ln = e - y * kNB1;
        const bool ok = n0 + ln < d.NZ;
        cp_async16z(stg + e, ok ? src + y * ystride + ln : Q1, ok);
      }
    }
    cp_async_commit();
  };
  issue(blockIdx.x);
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int qi = tile % nq, r = tile / nq, nb = r % nnb, kx = r / nnb, n0 = nb * kNB1;
    cp_async_wait<0>();
    __syncthreads();
    auto ld = [&](int ln, int y) -> double2 {
      const double2 v = stg[y * kNB1 + ln];
      return (n0 + ln == 0) ? cscale(v, 0.5) : v;
    };
    fft_pass_first<NF, P.r[0], false, kThreadsYF, kNB1, true>(A, kNB1, LS, ld);  // ends with a barrier
    issue(tile + gridDim.x);
    fft_passes<NF, 1, P.r[0], false, kThreadsYF, kNB1, kPlanYF>(A, kNB1, LS, py.tw);
    // two adjacent Chebyshev rows per thread: one 32-byte store
    for (int idx = threadIdx.x; idx < (kNB1 / 2) * NYA; idx += blockDim.x) {
      const int l0 = 2 * (idx % (kNB1 / 2)), ky = idx / (kNB1 / 2), n = n0 + l0;
      const double2 v0 = cscale(A[l0 * LS + ky], scale), v1 = cscale(A[(l0 + 1) * LS + ky], scale);
      double2* dst = qspec + (((size_t)qi * d.NXH + kx) * NYA + ky) * d.NZ + n;
      if (n + 1 < d.NZ && aligned32(dst)) {
        st32(dst, v0, v1);
      } else {
        if (n < d.NZ) dst[0] = v0;
        if (n + 1 < d.NZ) dst[1] = v1;
      }
    }
    __syncthreads();  // A is rewritten by the next tile's first pass
  }
  cp_async_wait<0>();
}

// remove_vertical_mean_of_quadratic_var (PL_IMEX_timestepping.f90:223-235)
__global__ void k_remove_zmean(Dims d, double2* qs) {
  const size_t col = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= (size_t)d.NXH * d.NYA) return;
  double2* s = qs + col * d.NZ;
  double2 acc = zero2();
  for (int q = 1; q <= d.NZ / 2 - 1; ++q) {
    const double c = 0.5 / (2.0 * q + 1.0) - 0.5 / (2.0 * q - 1.0);
    acc = csub(acc, cscale(s[2 * q], c));
  }
  s[0] = acc;
}

// ------------------------------------------------------------------------------
// NL assembly K_hat = sum_terms (i kx)^a (i ky)^b dsca trunc(I^Iz M^mz) qhat,
// inserted in the interleaved ordering (marching.f90:319-367); zero for dealiased
// modes and (0,0).  One warp per (kx,ky) system.
// ------------------------------------------------------------------------------
__global__ void __launch_bounds__(kWPB * 32) k_nl(NLArgs a) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int sid = blockIdx.x * kWPB + warp;
  const int nsys = a.d.NXH * a.d.NYA;
  if (sid >= nsys) return;
  const int kx = sid / a.d.NYA, ky = sid - kx * a.d.NYA;
  const bool act = a.act_index[sid] >= 0;
  double2 coef[kMaxGroups];
#pragma unroll
  for (int g = 0; g < kMaxGroups; ++g)
    coef[g] = (g < a.NL.ngroups) ? cmul(ipow(a.kx[kx], a.NL.gkx[g]), ipow(a.ky[ky], a.NL.gky[g])) : zero2();
  double2* out = a.Khat + (size_t)sid * a.T;
  const int NZ = a.d.NZ;
  for (int t = lane; t < a.T; t += 32) {
    double2 acc = zero2();
    for (int k = 0; act && k < a.NL.width; ++k) {
      const double v = a.NL.v(t, k);
      if (v == 0.0) break;  // slots are filled in order; exact zeros are not stored
      const int c = a.NL.col(t, k);
      const int qv = c / NZ, n = c - qv * NZ;
      const double2 qh = a.qspec[(((size_t)qv * a.d.NXH + kx) * a.d.NYA + ky) * NZ + n];
      double2 cv = coef[0];
      const int g = a.NL.grp(t, k);
#pragma unroll
      for (int gg = 1; gg < kMaxGroups; ++gg)
        if (g == gg) cv = coef[gg];
      acc = cadd(acc, cmul(cv, make_double2(v * qh.x, v * qh.y)));
    }
    out[t] = acc;
  }
}

// ------------------------------------------------------------------------------
// stage update and banded solve, one warp per (kx,ky) system
//   rhs = M field + sum_{j<i} dt a(i,j) Kstd_j + dt ahat(i+1,j) Khat_j + dt ahat(i+1,i) Khat_i
//   aux = E^{-1} rhs  (E = identity for dealiased modes; (0,0): M is empty)
//   Kstd_i = L aux    (zero for dealiased modes and (0,0))
// (marching.f90:16-29, 53-171; PL_algebra_z_3D.f90:218-243 zgbtrs semantics)
// ------------------------------------------------------------------------------
constexpr int kPF = 8;  // factor columns prefetched ahead

__device__ __forceinline__ double2 ell_row(const DevEll& op, int t, const double2* coef, const double2* x) {
  double2 acc = zero2();
#pragma unroll 4
  for (int k = 0; k < op.width; ++k) {
    const int cg = op.cg[(size_t)k * op.rows + t];
    const double v = op.val[(size_t)k * op.rows + t];
    const double2 xv = x[cg & 0xFFFFFF];
    acc = cadd(acc, cmul(coef[cg >> 24], make_double2(v * xv.x, v * xv.y)));
  }
  return acc;
}

// WIDE: bands of kl <= 63, kl + ku <= 127 (each lane holds two multipliers and
// four U entries of a column); otherwise kl <= 31, kl + ku <= 64
template <bool WIDE>
__global__ void __launch_bounds__(kWPB * 32) k_solve(SolveArgs a) {
  extern __shared__ double2 sm[];
  __shared__ double2 coefs[kWPB][2][kMaxGroups];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int sid = blockIdx.x * kWPB + warp;
  const int nsys = a.d.NXH * a.d.NYA;
  if (sid >= nsys) return;
  const int T = a.T;
  double2* b = sm + (size_t)warp * T;
  const int kx = sid / a.d.NYA, ky = sid - kx * a.d.NYA;
  const int act = a.act_index[sid];
  const bool origin = (kx == 0 && ky == 0);
  if (lane < kMaxGroups) {
    coefs[warp][0][lane] = (lane < a.M.ngroups) ? cmul(ipow(a.kx[kx], a.M.gkx[lane]), ipow(a.ky[ky], a.M.gky[lane])) : zero2();
    coefs[warp][1][lane] = (lane < a.L.ngroups) ? cmul(ipow(a.kx[kx], a.L.gkx[lane]), ipow(a.ky[ky], a.L.gky[lane])) : zero2();
  }
  __syncwarp();
  const double2* field = a.field + (size_t)sid * T;
  // ---- right-hand side
  for (int t = lane; t < T; t += 32) {
    double2 r = origin ? zero2() : ell_row(a.M, t, coefs[warp][0], field);
    for (int j = 0; j < a.nprev; ++j) {
      const double2 ks = a.Kstd[j][(size_t)sid * T + t];
      r = cadd(r, cscale(ks, a.ca[j]));
      const double2 kh = a.Khat[j][(size_t)sid * T + t];
      r = cadd(r, cscale(kh, a.ch[j]));
    }
    const double2 kh = a.Khat[a.nprev][(size_t)sid * T + t];
    r = cadd(r, cscale(kh, a.ch[a.nprev]));
    b[t] = r;
  }
  __syncwarp();
  if (act >= 0) {
    const int kl = a.kl, kv = a.kl + a.ku, ldab = a.ldab;
    const double2* ab = a.ab + (size_t)act * T * ldab;
    const unsigned char* dp = a.dpiv + (size_t)act * ((T + 7) & ~7);
    // ---- forward: apply row interchanges and L (zgbtrs, 'N', kl > 0)
    {
      double2 lr[kPF], lr2[WIDE ? kPF : 1];
#pragma unroll
      for (int q = 0; q < kPF; ++q) {
        lr[q] = (q < T - 1 && lane < kl) ? ab[(size_t)q * ldab + kv + 1 + lane] : zero2();
        if constexpr (WIDE) lr2[q] = (q < T - 1 && lane + 32 < kl) ? ab[(size_t)q * ldab + kv + 33 + lane] : zero2();
      }
      for (int j0 = 0; j0 < T - 1; j0 += kPF) {
#pragma unroll
        for (int q = 0; q < kPF; ++q) {
          const int j = j0 + q;
          if (j < T - 1) {
            const double2 l = lr[q];
            double2 l2 = zero2();
            const int jn = j + kPF;
            lr[q] = (jn < T - 1 && lane < kl) ? ab[(size_t)jn * ldab + kv + 1 + lane] : zero2();
            if constexpr (WIDE) {
              l2 = lr2[q];
              lr2[q] = (jn < T - 1 && lane + 32 < kl) ? ab[(size_t)jn * ldab + kv + 33 + lane] : zero2();
            }
            const int p = j + dp[j];
            if (p != j) {
              if (lane == 0) {
                double2 tmp = b[p];
                b[p] = b[j];
                b[j] = tmp;
              }
              __syncwarp();
            }
            const double2 bj = b[j];
            const int lm = min(kl, T - 1 - j);
            if (lane < lm) b[j + 1 + lane] = csub(b[j + 1 + lane], cmul(l, bj));
            if constexpr (WIDE)
              if (lane + 32 < lm) b[j + 33 + lane] = csub(b[j + 33 + lane], cmul(l2, bj));
            __syncwarp();
          }
        }
      }
    }
    // ---- backward: U x = y, U with kl+ku super-diagonals, diagonal stored as its reciprocal
    {
      constexpr int NU = WIDE ? 4 : 2;  // U entries per lane: offsets 1 + lane + 32 u
      double2 uu[NU][kPF], dg[kPF];
#pragma unroll
      for (int q = 0; q < kPF; ++q) {
        const int j = T - 1 - q;
        if (j >= 0) {
          const double2* col = ab + (size_t)j * ldab;
          dg[q] = col[kv];
#pragma unroll
          for (int u = 0; u < NU; ++u) uu[u][q] = (lane + 1 + 32 * u <= kv) ? col[kv - 1 - 32 * u - lane] : zero2();
        }
      }
      for (int j0 = T - 1; j0 >= 0; j0 -= kPF) {
#pragma unroll
        for (int q = 0; q < kPF; ++q) {
          const int j = j0 - q;
          if (j >= 0) {
            const double2 d = dg[q];
            double2 c[NU];
#pragma unroll
            for (int u = 0; u < NU; ++u) c[u] = uu[u][q];
            const int jn = j - kPF;
            if (jn >= 0) {
              const double2* col = ab + (size_t)jn * ldab;
              dg[q] = col[kv];
#pragma unroll
              for (int u = 0; u < NU; ++u) uu[u][q] = (lane + 1 + 32 * u <= kv) ? col[kv - 1 - 32 * u - lane] : zero2();
            }
            const double2 bj = cmul(b[j], d);
            __syncwarp();
            if (lane == 0) b[j] = bj;
#pragma unroll
            for (int u = 0; u < NU; ++u) {
              const int o = lane + 1 + 32 * u;
              if (o <= kv && j - o >= 0) b[j - o] = csub(b[j - o], cmul(c[u], bj));
            }
            __syncwarp();
          }
        }
      }
    }
  }
  // ---- outputs
  double2* out = a.out + (size_t)sid * T;
  bool bad = false;
  const bool zero_out = a.last_stage && (act < 0);
  for (int t = lane; t < T; t += 32) {
    const double2 v = zero_out ? zero2() : b[t];
    bad |= !(isfinite(v.x) && isfinite(v.y));
    out[t] = v;
  }
  if (a.Kstd_out) {
    double2* ko = a.Kstd_out + (size_t)sid * T;
    for (int t = lane; t < T; t += 32) ko[t] = (act >= 0) ? ell_row(a.L, t, coefs[warp][1], b) : zero2();
  }
  if (__any_sync(0xffffffffu, bad) && lane == 0) atomicOr(a.flags, 1u);
}

// ------------------------------------------------------------------------------
// factorisation of E = M + zsca L (zsca = -dt a11) with partial pivoting, one warp
// per active system, in place in LAPACK band storage (PL_IMEX_timestepping.f90:382-410;
// PL_algebra_z_3D.f90:245-276; the unblocked ZGBTF2 algorithm that ZGBTRF runs for
// kl < 32).  Pivot offsets are kept as bytes; U's diagonal is replaced by its reciprocal.
// ------------------------------------------------------------------------------
__device__ __forceinline__ double2 crecip(double2 p) {
  if (fabs(p.x) >= fabs(p.y)) {
    const double t = p.y / p.x, den = p.x + p.y * t;
    return make_double2(1.0 / den, -t / den);
  } else {
    const double t = p.x / p.y, den = p.y + p.x * t;
    return make_double2(t / den, -1.0 / den);
  }
}

// WIDE: kl <= 63 (two pivot candidates per lane); otherwise kl <= 31
template <bool WIDE>
__global__ void __launch_bounds__(kWPB * 32) k_factor(FactorArgs a) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int sys = blockIdx.x * kWPB + warp;
  if (sys >= a.nact) return;
  const int T = a.T, kl = a.kl, ku = a.ku, kv = kl + ku, ldab = a.ldab;
  const int sid = a.act_list[sys];
  const int kx = sid / a.d.NYA, ky = sid - kx * a.d.NYA;
  double2 cm[kMaxGroups], cl[kMaxGroups];
#pragma unroll
  for (int g = 0; g < kMaxGroups; ++g) {
    cm[g] = (g < a.M.ngroups) ? cmul(ipow(a.kx[kx], a.M.gkx[g]), ipow(a.ky[ky], a.M.gky[g])) : zero2();
    cl[g] = (g < a.L.ngroups) ? cmul(ipow(a.kx[kx], a.L.gkx[g]), ipow(a.ky[ky], a.L.gky[g])) : zero2();
  }
  double2* ab = a.ab + (size_t)sys * T * ldab;
  for (size_t e = lane; e < (size_t)T * ldab; e += 32) ab[e] = zero2();
  __syncwarp();
  // E(t,c) = M(t,c) + zsca * L(t,c); lane owns rows t = lane mod 32 (no write conflicts)
  for (int t = lane; t < T; t += 32) {
    for (int k = 0; k < a.M.width; ++k) {
      const double v = a.M.v(t, k);
      if (v == 0.0) continue;  // empty slot
      const int c = a.M.col(t, k), g = a.M.grp(t, k);
      double2 cv = zero2();
#pragma unroll
      for (int gg = 0; gg < kMaxGroups; ++gg)
        if (g == gg) cv = cm[gg];
      double2& dst = ab[(size_t)c * ldab + kv + t - c];
      dst = cadd(dst, cscale(cv, v));
    }
    for (int k = 0; k < a.L.width; ++k) {
      const double v = a.L.v(t, k);
      if (v == 0.0) continue;
      const int c = a.L.col(t, k), g = a.L.grp(t, k);
      double2 cv = zero2();
#pragma unroll
      for (int gg = 0; gg < kMaxGroups; ++gg)
        if (g == gg) cv = cl[gg];
      double2& dst = ab[(size_t)c * ldab + kv + t - c];
      dst = cadd(dst, cscale(cscale(cv, v), a.zsca));
    }
  }
  __syncwarp();
  int ju = 0, info = 0;
  for (int j = 0; j < T; ++j) {
    const int km = min(kl, T - 1 - j);
    // pivot: first index of the largest |re|+|im| among rows j..j+km
    double mag = -1.0;
    int idx = 1 << 30;
    if (lane <= km) {
      const double2 v = ab[(size_t)j * ldab + kv + lane];
      mag = fabs(v.x) + fabs(v.y);
      idx = lane;
    }
    if constexpr (WIDE) {
      if (lane + 32 <= km) {  // the later row wins only when strictly larger (first maximum)
        const double2 v = ab[(size_t)j * ldab + kv + lane + 32];
        const double m2 = fabs(v.x) + fabs(v.y);
        if (m2 > mag) { mag = m2; idx = lane + 32; }
      }
    }
    for (int o = 16; o > 0; o >>= 1) {
      const double m2 = __shfl_xor_sync(0xffffffffu, mag, o);
      const int i2 = __shfl_xor_sync(0xffffffffu, idx, o);
      if (m2 > mag || (m2 == mag && i2 < idx)) { mag = m2; idx = i2; }
    }
    const int jp = idx;
    if (lane == 0) a.dpiv[(size_t)sys * ((T + 7) & ~7) + j] = (unsigned char)jp;
    const double2 piv = ab[(size_t)j * ldab + kv + jp];
    if (piv.x == 0.0 && piv.y == 0.0) {
      if (info == 0) info = j + 1;
      continue;
    }
    ju = max(ju, min(j + ku + jp, T - 1));
    if (jp != 0) {
      for (int c = j + lane; c <= ju; c += 32) {
        double2* p1 = ab + (size_t)c * ldab + kv + j + jp - c;
        double2* p0 = ab + (size_t)c * ldab + kv + j - c;
        const double2 t0 = *p0;
        *p0 = *p1;
        *p1 = t0;
      }
      __syncwarp();
    }
    const double2 r = crecip(ab[(size_t)j * ldab + kv]);
    __syncwarp();
    if (km > 0) {
      for (int i = lane; i <= km; i += 32)
        if (i >= 1) {
          double2* m = ab + (size_t)j * ldab + kv + i;
          *m = cmul(*m, r);
        }
      __syncwarp();
      const int nc = ju - j;
      for (int e = lane; e < nc * km; e += 32) {
        const int c = j + 1 + e / km, i = 1 + e % km;
        const double2 mult = ab[(size_t)j * ldab + kv + i];
        const double2 rowv = ab[(size_t)c * ldab + kv + j - c];
        double2* dst = ab + (size_t)c * ldab + kv + j + i - c;
        *dst = csub(*dst, cmul(mult, rowv));
      }
    }
    __syncwarp();
    if (lane == 0) ab[(size_t)j * ldab + kv] = r;
    __syncwarp();
  }
  if (lane == 0) a.info[sys] = info;
}


// ------------------------------------------------------------------------------
// Real-scaled factorisation: E' = S_r E S_c with S_r = diag(-i on flagged
// equation rows), S_c = diag(+i on flagged variable columns) is real; the
// partial-pivoting choices equal those on E because |re|+|im| is unchanged by
// the +-i factors.  Real ZGBTF2-equivalent (DGBTF2), one warp per system, in place
// in LAPACK band storage; pivot offsets as bytes; U's diagonal as its reciprocal.
// ------------------------------------------------------------------------------
__device__ __forceinline__ double2 flip_row(double2 z, int f) { return f ? make_double2(z.y, -z.x) : z; }  // * (-i)
__device__ __forceinline__ double2 flip_col(double2 z, int f) { return f ? make_double2(-z.y, z.x) : z; }  // * (+i)

// With a class split (FactorArgs::ncls == 2) one warp factors one class of one
// system (blockIdx.y = class): the class's rows and columns in their original
// relative order, identity rows on padding positions, stored in the class's
// ldab rows of each column (column stride ncls * ldab).
__global__ void __launch_bounds__(kWPB * 32) k_factor_real(FactorArgs a) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int sys = blockIdx.x * kWPB + warp;
  if (sys >= a.nact) return;
  const int cls = blockIdx.y;
  const int T = a.Tc, kl = a.kl, ku = a.ku, kv = kl + ku, ldab = a.ldab;
  const size_t cstr = (size_t)a.ncls * ldab;  // column stride
  const int sid = a.act_list[sys];
  const int kx = sid / a.d.NYA, ky = sid - kx * a.d.NYA;
  double2 cm[kMaxGroups], cl[kMaxGroups];
#pragma unroll
  for (int g = 0; g < kMaxGroups; ++g) {
    cm[g] = (g < a.M.ngroups) ? cmul(ipow(a.kx[kx], a.M.gkx[g]), ipow(a.ky[ky], a.M.gky[g])) : zero2();
    cl[g] = (g < a.L.ngroups) ? cmul(ipow(a.kx[kx], a.L.gkx[g]), ipow(a.ky[ky], a.L.gky[g])) : zero2();
  }
  double* ab = a.abr + (size_t)sys * T * cstr + (size_t)cls * ldab;
  for (size_t e = lane; e < (size_t)T * ldab; e += 32) ab[(e / ldab) * cstr + e % ldab] = 0.0;
  __syncwarp();
  for (int i = lane; i < T; i += 32) {
    const int t = a.cls_row ? a.cls_row[cls * T + i] : i;  // equation row of class position i
    if (t < 0) {
      ab[(size_t)i * cstr + kv] = 1.0;  // identity padding
      continue;
    }
    const int rf = a.rowflip[t];
    for (int pass = 0; pass < 2; ++pass) {
      const DevEll& op = pass ? a.L : a.M;
      for (int k = 0; k < op.width; ++k) {
        const double v = op.v(t, k);
        if (v == 0.0) continue;  // empty slot
        const int c = op.col(t, k), g = op.grp(t, k);
        const int jc = a.col_pos ? a.col_pos[c] - cls * T : c;  // column in the class
        double2 cv = zero2();
#pragma unroll
        for (int gg = 0; gg < kMaxGroups; ++gg)
          if (g == gg) cv = pass ? cl[gg] : cm[gg];
        double2 z = cscale(cv, v);
        if (pass) z = cscale(z, a.zsca);
        z = flip_col(flip_row(z, rf), a.colflip[c]);
        ab[(size_t)jc * cstr + kv + i - jc] += z.x;
      }
    }
  }
  __syncwarp();
  unsigned char* dpiv = a.dpiv + ((size_t)sys * a.ncls + cls) * ((T + 7) & ~7);  // rows padded to 8 bytes
  int ju = 0, info = 0;
  for (int j = 0; j < T; ++j) {
    const int km = min(kl, T - 1 - j);
    double mag = -1.0;
    int idx = 1 << 30;
    if (lane <= km) {
      mag = fabs(ab[(size_t)j * cstr + kv + lane]);
      idx = lane;
    }
    for (int o = 16; o > 0; o >>= 1) {
      const double m2 = __shfl_xor_sync(0xffffffffu, mag, o);
      const int i2 = __shfl_xor_sync(0xffffffffu, idx, o);
      if (m2 > mag || (m2 == mag && i2 < idx)) { mag = m2; idx = i2; }
    }
    const int jp = idx;
    if (lane == 0) dpiv[j] = (unsigned char)jp;
    const double piv = ab[(size_t)j * cstr + kv + jp];
    if (piv == 0.0) {
      if (info == 0) info = j + 1;
      continue;
    }
    ju = max(ju, min(j + ku + jp, T - 1));
    if (jp != 0) {
      for (int c = j + lane; c <= ju; c += 32) {
        double* p1 = ab + (size_t)c * cstr + kv + j + jp - c;
        double* p0 = ab + (size_t)c * cstr + kv + j - c;
        const double t0 = *p0;
        *p0 = *p1;
        *p1 = t0;
      }
      __syncwarp();
    }
    const double r = 1.0 / ab[(size_t)j * cstr + kv];
    __syncwarp();
    if (km > 0) {
      if (lane >= 1 && lane <= km) ab[(size_t)j * cstr + kv + lane] *= r;
      __syncwarp();
      const int nc = ju - j;
      for (int e = lane; e < nc * km; e += 32) {
        const int c = j + 1 + e / km, i = 1 + e % km;
        ab[(size_t)c * cstr + kv + j + i - c] -= ab[(size_t)j * cstr + kv + i] * ab[(size_t)c * cstr + kv + j - c];
      }
    }
    __syncwarp();
    if (lane == 0) ab[(size_t)j * cstr + kv] = r;
    __syncwarp();
  }
  if (lane == 0 && info) atomicMax(a.info + sys, info);
}

// ------------------------------------------------------------------------------
// Stage update + banded solve with real-scaled factors, one warp per system,
// no shared-memory vectors: the right-hand side and the intermediate solutions
// pass through the work array (L2-resident), while the active part of the
// band lives in registers, each lane owning the positions p = lane (mod 32):
//   forward  window [j, j+kl] (kl <= 31), one register per lane
//   backward window [j-kv, j] (kv <= 63), two registers per lane
// so a column step moves only the pivot value between lanes.  Factor columns
// reach the lanes through a per-warp shared-memory ring filled by cp.async.
// ------------------------------------------------------------------------------
constexpr int kWPBr = 4;   // warps per CTA
constexpr int kCW = 8;     // factor columns per ring chunk (divides 32)
constexpr int kNBUF = 4;   // ring chunks per warp

__device__ __forceinline__ double2 shfl2(double2 v, int src) {
  return make_double2(__shfl_sync(0xffffffffu, v.x, src), __shfl_sync(0xffffffffu, v.y, src));
}

// H = lanes per system class: H = 32 for an unsplit system, H = 16 for a class
// split, the two classes of one system side by side in the two half-warps, in
// lockstep over their Tc columns (positions p = lane (mod H) of the half; the
// window bounds become kl <= H-1 and kl+ku <= 2H-1).
template <int H>
__global__ void __launch_bounds__(kWPBr * 32) k_subst_real(SolveArgs a) {
  constexpr int NC = 32 / H;            // classes per warp
  constexpr int LH = (H == 32) ? 5 : 4;  // log2(H)
  extern __shared__ double smr[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int hl = lane & (H - 1);         // lane within the class's half
  const int cls = lane >> LH;
  const int hb = lane - hl;              // first lane of the half
  const int act = blockIdx.x * kWPBr + warp;  // active systems only
  if (act >= a.nact) return;
  const int T = a.Tc;
  const int sid = a.act_list[act];
  double2* x = a.work + (size_t)sid * a.wst + (size_t)cls * T;  // right-hand side in, solution out
  {
    const int kl = a.kl, kv = a.kl + a.ku, ldab = a.ldab;
    const size_t cstr = (size_t)NC * ldab;  // factor column stride (both classes)
    const double* ab = a.abr + (size_t)act * T * cstr;
    const unsigned char* dp = a.dpiv + ((size_t)act * NC + cls) * ((T + 7) & ~7);
    const unsigned char* cflip = a.colflip_cls + (size_t)cls * T;
    // Factor columns stream through a per-warp shared-memory ring (kNBUF chunks
    // of kCW columns) with cp.async, kNBUF-1 chunks ahead of the sweep; the
    // forward sweep copies only the L rows of each column, the backward sweep
    // only the U rows.  (ldab is even, so both row ranges are 16-byte aligned.)
    double* ring = smr + (size_t)warp * kNBUF * kCW * a.ring_cols;
    const int rc = a.ring_cols / NC;                  // ring doubles per class and column
    const int u_rows = (kv + 2) & ~1;                 // rows [0, u_rows) hold U (+ maybe one L row)
    const int l_row0 = (kv + 1) & ~1;                 // rows [l_row0, l_row1) hold L
    const int l_rows = ((kv + 1 + kl + 1) & ~1) - l_row0;
    // ================= forward: P and L =================
    // lane l owns the positions p = l (mod H); the active window is [j, j+kl].
    // Vector traffic moves in blocks of H columns: the owner of column j takes
    // the new position j+H (loaded one block ahead) and parks y_j until the
    // block's coalesced store.
    {
      const int nchunks = (T - 1 + kCW - 1) / kCW;
      auto issue = [&](int c) {  // columns [c*kCW, min(T-1, c*kCW+kCW)) of L
        if (c < nchunks) {
          const int j0 = c * kCW, nc = min(kCW, T - 1 - j0);
          double* dst = ring + (size_t)(c % kNBUF) * kCW * a.ring_cols;
          const int per = l_rows / 2;  // 16-byte pieces per column and class
          for (int e = lane; e < nc * NC * per; e += 32) {
            const int q = e / (NC * per), rem = e - q * (NC * per), cc = rem / per, r = rem - cc * per;
            cp_async16(dst + q * a.ring_cols + cc * rc + 2 * r, ab + (size_t)(j0 + q) * cstr + cc * ldab + l_row0 + 2 * r);
          }
        }
        cp_async_commit();
      };
#pragma unroll
      for (int c = 0; c < kNBUF - 1; ++c) issue(c);
      double2 w = (hl < T) ? x[hl] : zero2();
      double2 incCur = (H + hl < T) ? x[H + hl] : zero2();
      double2 incNext = zero2(), ysave = zero2();
      // pivot offsets of a chunk as two 32-bit words, uniform over the half (rows padded to 8 bytes)
      uint2 pw = *reinterpret_cast<const uint2*>(dp);
      for (int c = 0; c < nchunks; ++c) {
        const int j0 = c * kCW;
        if ((j0 & (H - 1)) == 0)  // new block of H columns: next block's incoming values
          incNext = (j0 + 2 * H + hl < T) ? x[j0 + 2 * H + hl] : zero2();
        const uint2 pwc = pw;
        if (c + 1 < nchunks) pw = *reinterpret_cast<const uint2*>(dp + j0 + kCW);
        __syncwarp();
        issue(c + kNBUF - 1);
        cp_async_wait<kNBUF - 1>();
        __syncwarp();
        const double* cb = ring + (size_t)(c % kNBUF) * kCW * a.ring_cols + cls * rc;
#pragma unroll
        for (int q = 0; q < kCW; ++q) {
          const int j = j0 + q;
          if (j < T - 1) {
            const int src = hb + (j & (H - 1));
            const int i = (hl - j) & (H - 1);
            const int lm = min(kl, T - 1 - j);
            const double lv = (i >= 1 && i <= lm) ? cb[q * a.ring_cols + (kv + i - l_row0)] : 0.0;
            const int jp = ((q < 4 ? pwc.x : pwc.y) >> (8 * (q & 3))) & 0xFF;
            // Row interchange j <-> j+jp and broadcast of the pivot row in one shuffle:
            // the owner of row j+jp fetches row j (its new content), every other lane
            // fetches the pivot row; the owner of j+jp already holds the pivot value.
            const int r2 = hb + ((j + jp) & (H - 1));
            const bool mine = (jp != 0 && lane == r2);
            const double2 got = shfl2(w, mine ? src : r2);
            const double2 bj = mine ? w : got;
            if (lane == src || mine) w = got;
            w.x -= lv * bj.x;  // zero multiplier outside rows j+1..j+lm
            w.y -= lv * bj.y;
            if (lane == src) {
              ysave = w;
              w = incCur;
            }
            if ((j & (H - 1)) == H - 1) {  // end of a block of H columns
              x[j - (H - 1) + hl] = ysave;
              incCur = incNext;
            }
          }
        }
      }
      cp_async_wait<0>();
      // the last (partial) block of y values and y[T-1]
      const int base = ((T - 1) >> LH) << LH;
      if ((T - 1) & (H - 1)) {
        if (base + hl <= T - 2) x[base + hl] = ysave;
      }
      if (hl == ((T - 1) & (H - 1))) x[T - 1] = w;
    }
    __syncwarp();
    // ================= backward: U (kl+ku super-diagonals, reciprocal diagonal) =================
    // lane l owns p = l (mod H) in two registers: w0 for (p/H) even, w1 for odd.
    // Blocks of H columns j = T-1-H*b-s; the owner of j takes position j-2H.
    {
      double2 w0 = zero2(), w1 = zero2();
      {
        const int ih = (T - 1 - hl) & (H - 1), ph = T - 1 - ih, pl = ph - H;
        if (ph >= 0) { if ((ph >> LH) & 1) w1 = x[ph]; else w0 = x[ph]; }
        if (pl >= 0) { if ((pl >> LH) & 1) w1 = x[pl]; else w0 = x[pl]; }
      }
      const int nchunks = (T + kCW - 1) / kCW;  // chunk c: columns T-1-c*kCW-q, q < kCW
      auto issue = [&](int c) {
        if (c < nchunks) {
          const int jhi = T - 1 - c * kCW, jlo = max(0, jhi - kCW + 1), nc = jhi - jlo + 1;
          double* dst = ring + (size_t)(c % kNBUF) * kCW * a.ring_cols;
          const int per = u_rows / 2;
          for (int e = lane; e < nc * NC * per; e += 32) {
            const int q = e / (NC * per), rem = e - q * (NC * per), cc = rem / per, r = rem - cc * per;  // q counts down from jhi
            cp_async16(dst + q * a.ring_cols + cc * rc + 2 * r, ab + (size_t)(jhi - q) * cstr + cc * ldab + 2 * r);
          }
        }
        cp_async_commit();
      };
      __syncwarp();
#pragma unroll
      for (int c = 0; c < kNBUF - 1; ++c) issue(c);
      auto own_col = [&](int b) {  // column of block b finished by this lane (may be < 0)
        const int top = T - 1 - H * b;
        return top - ((top - hl) & (H - 1));
      };
      int jl = own_col(0);
      double2 incCur = (jl - 2 * H >= 0) ? x[jl - 2 * H] : zero2();
      int cfCur = (jl >= 0) ? cflip[jl] : 0;
      double2 incNext = zero2(), xsave = zero2();
      int cfNext = 0, jn = jl;
      for (int c = 0; c < nchunks; ++c) {
        const int k0 = c * kCW;  // steps taken before this chunk
        if ((k0 & (H - 1)) == 0) {
          jn = own_col((k0 >> LH) + 1);
          incNext = (jn - 2 * H >= 0) ? x[jn - 2 * H] : zero2();
          cfNext = (jn >= 0) ? cflip[jn] : 0;
        }
        __syncwarp();
        issue(c + kNBUF - 1);
        cp_async_wait<kNBUF - 1>();
        __syncwarp();
        const double* cb = ring + (size_t)(c % kNBUF) * kCW * a.ring_cols + cls * rc;
#pragma unroll
        for (int q = 0; q < kCW; ++q) {
          const int k = k0 + q;
          const int j = T - 1 - k;
          if (j >= 0) {
            const int src = hb + (j & (H - 1)), sel = (j >> LH) & 1;
            const double* col = cb + q * a.ring_cols;
            const int ih = (j - hl) & (H - 1), il = ih + H;
            const double h = (ih >= 1 && ih <= kv) ? col[kv - ih] : 0.0;
            const double l_ = (il <= kv) ? col[kv - il] : 0.0;
            const double d = col[kv];
            const double2 yj = shfl2(sel ? w1 : w0, src);
            const double2 xj = make_double2(yj.x * d, yj.y * d);
            const int hreg = ((j - ih) >> LH) & 1;
            if (hreg) { w1.x -= h * xj.x; w1.y -= h * xj.y; w0.x -= l_ * xj.x; w0.y -= l_ * xj.y; }
            else      { w0.x -= h * xj.x; w0.y -= h * xj.y; w1.x -= l_ * xj.x; w1.y -= l_ * xj.y; }
            if (lane == src) {
              xsave = flip_col(xj, cfCur);
              if (sel) w1 = incCur; else w0 = incCur;
            }
            if ((k & (H - 1)) == H - 1) {  // end of a block of H columns
              if (jl >= 0) x[jl] = xsave;
              jl = jn;
              incCur = incNext;
              cfCur = cfNext;
            }
          }
        }
      }
      cp_async_wait<0>();
      if ((T & (H - 1)) != 0 && jl >= 0) x[jl] = xsave;  // the last (partial) block
    }
  }
  __syncwarp();
}


// ------------------------------------------------------------------------------
// Thread-per-block solve of the independent blocks (class split).  Block
// b = ncls * act + class is handled by one thread; the 32 blocks of a group lie
// side by side in memory (abr[((g Tc + j) ldab + r) 32 + lane]), so every factor
// row, pivot byte and vector entry a warp touches in one step is one contiguous
// 256 / 32 / 512-byte row.  A thread keeps its band window in its own
// shared-memory column (slot stride kTpbThreads), where the data-dependent
// row interchange is a plain indexed access.
// ------------------------------------------------------------------------------
constexpr int kTpbThreads = 128;

// DGBTF2 on one block, in the interleaved layout: the algorithm, pivot choice
// and update order of k_factor_real.
// Assembly of block b (system b / ncls, class b % ncls) of M - dt a(0,0) L into
// its interleaved band storage: zero fill, then every operator entry added in
// row order (M before L, slots in order).
// G: the monomial groups the coefficient registers hold (>= the operators' ngroups)
template <int G = kMaxGroups>
__device__ void assemble_tpb(const FactorArgs& a, int b) {
  const int sys = b / a.ncls, cls = b - sys * a.ncls;
  const int T = a.Tc, kl = a.kl, ku = a.ku, kv = kl + ku, ldab = a.ldab;
  const int sid = a.act_list[sys];
  const int kx = sid / a.d.NYA, ky = sid - kx * a.d.NYA;
  double2 cm[G], cl[G];
#pragma unroll
  for (int g = 0; g < G; ++g) {
    cm[g] = (g < a.M.ngroups) ? cmul(ipow(a.kx[kx], a.M.gkx[g]), ipow(a.ky[ky], a.M.gky[g])) : zero2();
    cl[g] = (g < a.L.ngroups) ? cmul(ipow(a.kx[kx], a.L.gkx[g]), ipow(a.ky[ky], a.L.gky[g])) : zero2();
  }
  double* F = a.abr + (size_t)(b >> 5) * T * ldab * 32 + (b & 31);
  auto at = [&](int j, int r) -> double& { return F[((size_t)j * ldab + r) * 32]; };
  for (int j = 0; j < T; ++j)
    for (int r = 0; r < ldab; ++r) at(j, r) = 0.0;
  for (int i = 0; i < T; ++i) {
    const int t = a.cls_row[cls * T + i];  // equation row of class position i
    if (t < 0) {
      at(i, kv) = 1.0;  // identity padding
      continue;
    }
    const int rf = a.rowflip[t];
    for (int pass = 0; pass < 2; ++pass) {
      const DevEll& op = pass ? a.L : a.M;
      for (int k = 0; k < op.width; ++k) {
        const double v = op.v(t, k);
        if (v == 0.0) continue;  // empty slot
        const int c = op.col(t, k), g = op.grp(t, k);
        const int jc = a.col_pos[c] - cls * T;  // column in the class
        double2 cv = zero2();
#pragma unroll
        for (int gg = 0; gg < G; ++gg)
          if (g == gg) cv = pass ? cl[gg] : cm[gg];
        double2 z = cscale(cv, v);
        if (pass) z = cscale(z, a.zsca);
        z = flip_col(flip_row(z, rf), a.colflip[c]);
        at(jc, kv + i - jc) += z.x;
      }
    }
  }
}

template <int G>
__global__ void __launch_bounds__(kTpbThreads) k_assemble_tpb(FactorArgs a) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b < a.ncls * a.nact) assemble_tpb<G>(a, b);
}

__global__ void __launch_bounds__(kTpbThreads) k_factor_tpb(FactorArgs a) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= a.ncls * a.nact) return;
  assemble_tpb(a, b);
  const int sys = b / a.ncls;
  const int T = a.Tc, kl = a.kl, ku = a.ku, kv = kl + ku, ldab = a.ldab;
  double* F = a.abr + (size_t)(b >> 5) * T * ldab * 32 + (b & 31);
  auto at = [&](int j, int r) -> double& { return F[((size_t)j * ldab + r) * 32]; };
  unsigned char* P = a.dpiv + (size_t)(b >> 5) * T * 32 + (b & 31);
  int ju = 0, info = 0;
  for (int j = 0; j < T; ++j) {
    const int km = min(kl, T - 1 - j);
    int jp = 0;
    double mag = fabs(at(j, kv));
    for (int i = 1; i <= km; ++i) {
      const double m2 = fabs(at(j, kv + i));
      if (m2 > mag) { mag = m2; jp = i; }  // first maximum
    }
    P[(size_t)j * 32] = (unsigned char)jp;
    if (at(j, kv + jp) == 0.0) {
      if (info == 0) info = j + 1;
      continue;
    }
    ju = max(ju, min(j + ku + jp, T - 1));
    if (jp != 0) {
      for (int c = j; c <= ju; ++c) {
        double& p1 = at(c, kv + j + jp - c);
        double& p0 = at(c, kv + j - c);
        const double t0 = p0;
        p0 = p1;
        p1 = t0;
      }
    }
    const double r = 1.0 / at(j, kv);
    if (km > 0) {
      for (int i = 1; i <= km; ++i) at(j, kv + i) *= r;
      for (int c = j + 1; c <= ju; ++c) {
        const double u = at(c, kv + j - c);
        for (int i = 1; i <= km; ++i) at(c, kv + j + i - c) -= at(j, kv + i) * u;
      }
    }
    at(j, kv) = r;
  }
  if (info) atomicMax(a.info + sys, info);
}

// DGBTF2 on one block (after k_assemble_tpb) with its active band columns in
// shared memory: the algorithm, pivot choice and update order of k_factor_tpb
// (the same factors bit for bit), but every factor entry is read from and
// written to global memory once instead of being updated there up to kl times.
// At step j the window holds columns j .. j + W - 1 (W = kl + ku + 1: a step
// touches columns j .. ju, and ju <= j + ku + kl) and column j + W is in
// flight (cp.async, issued one step ahead into the slot column j - 1 left): a
// circular buffer of W + 1 slots.  Column j, final after step j, is written
// back in place.  Each thread's slots are (W + 1) ldab doubles in its own column
// of shared memory (slot stride blockDim.x <= 32), so the warp's accesses are
// conflict-free and its global accesses the 256-byte rows of the interleaved
// layout.  A step's multipliers and each updated column segment are staged in
// registers (kl <= kFacKl), so that its shared-memory loads issue together.
constexpr int kFacKl = 16;
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__global__ void __launch_bounds__(32) k_factor_win(FactorArgs a) {
  extern __shared__ double fwin[];
  const int NT = blockDim.x;
  const int b = blockIdx.x * NT + threadIdx.x;
  if (b >= a.ncls * a.nact) return;  // no barriers below
  const int sys = b / a.ncls;
  const int T = a.Tc, kl = a.kl, ku = a.ku, kv = kl + ku, ldab = a.ldab, W = kl + ku + 1, W1 = W + 1;
  double* F = a.abr + (size_t)(b >> 5) * T * ldab * 32 + (b & 31);
  double* wz = fwin + threadIdx.x;
  int j0 = 0, s0 = 0;  // the window's first column and its slot
  auto slot = [&](int c) { const int q = s0 + (c - j0); return q >= W1 ? q - W1 : q; };
  auto at = [&](int c, int r) -> double& { return wz[(slot(c) * ldab + r) * NT]; };
  auto fetch = [&](int c, int sl) {  // column c of the block into slot sl
    if (c < T) {
      const double* src = F + (size_t)c * ldab * 32;
      double* dst = wz + (size_t)sl * ldab * NT;
      for (int r = 0; r < ldab; ++r) cp_async8(dst + r * NT, src + (size_t)r * 32);
    }
  };
  for (int c = 0; c < W; ++c) fetch(c, c);
  cp_async_commit();
  unsigned char* P = a.dpiv + (size_t)(b >> 5) * T * 32 + (b & 31);
  int ju = 0, info = 0;
  for (int j = 0; j < T; ++j) {
    j0 = j;
    fetch(j + W, s0 == 0 ? W1 - 1 : s0 - 1);  // the slot column j - 1 left (the spare at j = 0)
    cp_async_commit();
    cp_async_wait<1>();  // columns up to j + W - 1 have landed
    const int km = min(kl, T - 1 - j);
    int jp = 0;
    double mag = fabs(at(j, kv));
    for (int i = 1; i <= km; ++i) {
      const double m2 = fabs(at(j, kv + i));
      if (m2 > mag) { mag = m2; jp = i; }  // first maximum
    }
    P[(size_t)j * 32] = (unsigned char)jp;
    if (at(j, kv + jp) == 0.0) {
      if (info == 0) info = j + 1;
    } else {
      ju = max(ju, min(j + ku + jp, T - 1));
      if (jp != 0) {
        for (int c = j; c <= ju; ++c) {
          double& p1 = at(c, kv + j + jp - c);
          double& p0 = at(c, kv + j - c);
          const double t0 = p0, t1 = p1;
          p0 = t1;
          p1 = t0;
        }
      }
      const double r = 1.0 / at(j, kv);
      if (km > 0) {
        double m[kFacKl];
        double* cj = wz + ((size_t)s0 * ldab + kv + 1) * NT;
#pragma unroll
        for (int i = 0; i < kFacKl; ++i) m[i] = (i < km) ? cj[i * NT] : 0.0;
#pragma unroll
        for (int i = 0; i < kFacKl; ++i)
          if (i < km) {
            m[i] *= r;
            cj[i * NT] = m[i];
          }
        for (int c = j + 1; c <= ju; ++c) {
          double* col = wz + ((size_t)slot(c) * ldab + kv + j - c) * NT;
          double x[kFacKl + 1];
#pragma unroll
          for (int i = 0; i <= kFacKl; ++i) x[i] = (i <= km) ? col[i * NT] : 0.0;
#pragma unroll
          for (int i = 0; i < kFacKl; ++i)
            if (i < km) col[(1 + i) * NT] = x[1 + i] - m[i] * x[0];
        }
      }
      at(j, kv) = r;
    }
    // column j is final
    const double* cw = wz + (size_t)s0 * ldab * NT;
    double* dst = F + (size_t)j * ldab * 32;
    for (int q = 0; q < ldab; ++q) dst[(size_t)q * 32] = cw[q * NT];
    s0 = (s0 + 1 == W1) ? 0 : s0 + 1;
  }
  cp_async_wait<0>();
  if (info) atomicMax(a.info + sys, info);
}

// Band rows that are nonzero in any block, per class column: one warp per
// (group, column) tests the 32 blocks of its group row by row (lanes beyond
// the last block count as zero).
__global__ void __launch_bounds__(256) k_mask_cols(FactorArgs a) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int g = blockIdx.x, j = blockIdx.y * 8 + w;
  const int T = a.Tc, ldab = a.ldab;
  if (j >= T) return;
  const bool ok = g * 32 + lane < a.ncls * a.nact;
  const double* F = a.abr + ((size_t)g * T + j) * ldab * 32 + lane;
  unsigned long long bits = 0;
  for (int r = 0; r < ldab; ++r) {
    const double v = ok ? F[(size_t)r * 32] : 0.0;
    if (__any_sync(0xffffffffu, v != 0.0)) bits |= 1ull << r;
  }
  if (lane == 0 && bits) atomicOr(a.cmask + j, bits);
}
// lmask / umask from cmask (see FactorArgs)
__global__ void k_mask_rows(FactorArgs a) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  const int T = a.Tc, kl = a.kl, kv = a.kl + a.ku;
  if (j >= T) return;
  a.lmask[j] = (unsigned)((a.cmask[j] >> (kv + 1)) & ((1ull << kl) - 1));
  unsigned u = 0;
  for (int i = 0; i < kv; ++i)
    if (j + 1 + i < T && ((a.cmask[j + 1 + i] >> (kv - 1 - i)) & 1ull)) u |= 1u << i;
  a.umask[j] = u;
}

// Forward (P, L: the column sweep with the row interchanges interleaved, as the
// reference's band solve) then backward (U, row form: each x_j subtracts the
// known x_{j+i} in decreasing column order, the order in which the column sweep
// reaches it) for one block.  The band is compile-time (kl = KL, kl + ku = KV,
// column stride LD = ldab), so every factor offset is an immediate from one
// per-column pointer; each step's factor values are loaded one step ahead.
// Band entries outside the matrix are stored zeros, so the forward sweep runs
// unpredicated (it only touches dead window slots near the end); the backward
// rows within KV of the last column take the guarded loop.
// The substitution of block b of the system described by a; win is this
// thread's band-window column in shared memory (slot stride kTpbThreads).
template <int KL, int KV, int LD>
__device__ __forceinline__ void subst_tpb_block(const SolveArgs& a, int b, double2* win) {
  constexpr int W1 = (KL + 2 <= 16) ? 16 : 32;  // power of 2 >= KL + 2
  constexpr int W2 = KV + 1;
  constexpr int S = kTpbThreads;                // slot stride
  constexpr size_t CS = (size_t)LD * 32;        // column stride (doubles)
  const int T = a.Tc;
  const int cls = b % a.ncls;
  const size_t gb = (size_t)(b >> 5) * T;
  const double* F = a.abr + gb * CS + (b & 31);
  const unsigned char* P = a.dpiv + gb * 32 + (b & 31);
  double2* X = a.work2 + gb * 32 + (b & 31);
  const unsigned char* cflip = a.colflip_cls + (size_t)cls * T;
  const int* ccol = a.cls_col + (size_t)cls * T;
  double2* out = a.out + (size_t)a.act_list[b / a.ncls] * a.T;  // this system's stage output
  bool bad = false;
  // ---- forward: positions j..j+KL in slots p mod W1 ----
  for (int p = 0; p <= KL && p < T; ++p) win[(p & (W1 - 1)) * S] = X[(size_t)p * 32];
  // L rows / U entries that are zero in every block are not loaded
  const unsigned* lmask = a.lmask;
  const unsigned* umask = a.umask;
  if (T > 1) {
    double lv[KL], lvn[KL];
    int jpn = P[0];
    double2 incn = (KL + 1 < T) ? X[(size_t)(KL + 1) * 32] : zero2();
    {
      const unsigned lm = lmask ? lmask[0] : ~0u;
#pragma unroll
      for (int i = 0; i < KL; ++i) lvn[i] = ((lm >> i) & 1u) ? F[(KV + 1 + i) * 32] : 0.0;
    }
    for (int j = 0; j < T - 1; ++j) {
#pragma unroll
      for (int i = 0; i < KL; ++i) lv[i] = lvn[i];
      const int jp = jpn;
      const double2 inc = incn;
      if (j + 1 < T - 1) {  // next column's multipliers, pivot and incoming entry
        const double* Fn = F + (size_t)(j + 1) * CS;
        const unsigned lm = lmask ? lmask[j + 1] : ~0u;
#pragma unroll
        for (int i = 0; i < KL; ++i) lvn[i] = ((lm >> i) & 1u) ? Fn[(KV + 1 + i) * 32] : 0.0;
        jpn = P[(size_t)(j + 1) * 32];
        incn = (j + KL + 2 < T) ? X[(size_t)(j + KL + 2) * 32] : zero2();
      }
      const int s0 = j & (W1 - 1);
      const int sp = (j + jp) & (W1 - 1);
      const double2 bj = win[sp * S];
      if (jp) win[sp * S] = win[s0 * S];
#pragma unroll
      for (int i = 0; i < KL; ++i) {
        const int sl = (s0 + 1 + i) & (W1 - 1);
        double2 w = win[sl * S];
        w.x -= lv[i] * bj.x;
        w.y -= lv[i] * bj.y;
        win[sl * S] = w;
      }
      X[(size_t)j * 32] = bj;
      if (j + KL + 1 < T) win[((j + KL + 1) & (W1 - 1)) * S] = inc;
    }
  }
  if (T > 0) X[(size_t)(T - 1) * 32] = win[((T - 1) & (W1 - 1)) * S];
  // ---- backward: x_{j+1}..x_{j+KV} in slots p mod W2 ----
  int sj = (T - 1) % W2;  // slot of position j
  int j = T - 1;
  for (; j >= 0 && j + KV >= T; --j) {  // rows within KV of the end
    const double* Fj = F + (size_t)j * CS;
    double2 acc = X[(size_t)j * 32];
    for (int i = T - 2 - j; i >= 0; --i) {
      int sl = sj + 1 + i;
      if (sl >= W2) sl -= W2;
      const double u = Fj[((1 + i) * LD + KV - 1 - i) * 32];
      const double2 xv = win[sl * S];
      acc.x -= u * xv.x;
      acc.y -= u * xv.y;
    }
    const double dinv = Fj[KV * 32];  // U's diagonal is stored as its reciprocal
    const double2 xj = make_double2(acc.x * dinv, acc.y * dinv);
    win[sj * S] = xj;
    {  // the solution, scaled back, straight into the stage output (original order)
      const int t = ccol[j];
      if (t >= 0) {
        const double2 xo = flip_col(xj, cflip[j]);
        bad |= !(isfinite(xo.x) && isfinite(xo.y));
        out[t] = xo;
      }
    }
    sj = (sj == 0) ? W2 - 1 : sj - 1;
  }
  if (j >= 0) {
    double u[KV], un[KV];
    double dinv, dinvn;
    double2 yn;
    {
      const double* Fj = F + (size_t)j * CS;
      const unsigned um = umask ? umask[j] : ~0u;
#pragma unroll
      for (int i = 0; i < KV; ++i) un[i] = ((um >> i) & 1u) ? Fj[((1 + i) * LD + KV - 1 - i) * 32] : 0.0;
      dinvn = Fj[KV * 32];
      yn = X[(size_t)j * 32];
    }
    for (; j >= 0; --j) {
#pragma unroll
      for (int i = 0; i < KV; ++i) u[i] = un[i];
      dinv = dinvn;
      double2 acc = yn;
      if (j > 0) {  // next row (j - 1)
        const double* Fn = F + (size_t)(j - 1) * CS;
        const unsigned um = umask ? umask[j - 1] : ~0u;
#pragma unroll
        for (int i = 0; i < KV; ++i) un[i] = ((um >> i) & 1u) ? Fn[((1 + i) * LD + KV - 1 - i) * 32] : 0.0;
        dinvn = Fn[KV * 32];
        yn = X[(size_t)(j - 1) * 32];
      }
#pragma unroll
      for (int i = KV - 1; i >= 0; --i) {
        int sl = sj + 1 + i;
        if (sl >= W2) sl -= W2;
        const double2 xv = win[sl * S];
        acc.x -= u[i] * xv.x;
        acc.y -= u[i] * xv.y;
      }
      const double2 xj = make_double2(acc.x * dinv, acc.y * dinv);
      win[sj * S] = xj;
      {  // the solution, scaled back, straight into the stage output (original order)
        const int t = ccol[j];
        if (t >= 0) {
          const double2 xo = flip_col(xj, cflip[j]);
          bad |= !(isfinite(xo.x) && isfinite(xo.y));
          out[t] = xo;
        }
      }
      sj = (sj == 0) ? W2 - 1 : sj - 1;
    }
  }
  // non-finite check (no warp-collective operation: lanes of a partial warp returned early)
  if (bad) atomicOr(a.flags, 1u);
}

template <int KL, int KV, int LD>
__global__ void __launch_bounds__(kTpbThreads) k_subst_tpb(SolveArgs a) {
  extern __shared__ double2 swin[];
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= a.nblk) return;  // no warp-collective operations below
  subst_tpb_block<KL, KV, LD>(a, b, swin + threadIdx.x);
}

// The substitutions of many systems (the members of an ensemble) in one
// persistent launch: thread slots walk the concatenated block range of all
// members (member m owns blocks [prefix[m], prefix[m+1])) with a grid stride;
// each block runs exactly the arithmetic of k_subst_tpb.
template <int KL, int KV, int LD>
__global__ void __launch_bounds__(kTpbThreads) k_subst_tpb_multi(const SolveArgs* args, const long long* prefix,
                                                                 int nmem, long long total) {
  extern __shared__ double2 swin[];
  for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x; g < total;
       g += (long long)gridDim.x * blockDim.x) {
    int lo = 0, hi = nmem - 1;  // member m with prefix[m] <= g < prefix[m+1]
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (prefix[mid] <= g) lo = mid;
      else hi = mid - 1;
    }
    subst_tpb_block<KL, KV, LD>(args[lo], (int)(g - prefix[lo]), swin + threadIdx.x);
  }
}

// The same solve for any band within (KL, KV) = (15, 31), kl and ku read at run time.
template <int KL, int KV>
__global__ void __launch_bounds__(kTpbThreads) k_subst_tpb_rt(SolveArgs a) {
  constexpr int W1 = (KL + 2 <= 16) ? 16 : 32;  // power of 2 >= KL + 2
  constexpr int W2 = KV + 1;
  constexpr int S = kTpbThreads;                // slot stride
  extern __shared__ double2 swin[];
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= a.nblk) return;  // no warp-collective operations below
  const int T = a.Tc, kl = a.kl, kv = a.kl + a.ku, ldab = a.ldab;
  const int cls = b % a.ncls;
  const size_t gb = (size_t)(b >> 5) * T;
  const double* F = a.abr + gb * ldab * 32 + (b & 31);
  const unsigned char* P = a.dpiv + gb * 32 + (b & 31);
  double2* X = a.work2 + gb * 32 + (b & 31);
  const unsigned char* cflip = a.colflip_cls + (size_t)cls * T;
  const int* ccol = a.cls_col + (size_t)cls * T;
  double2* out = a.out + (size_t)a.act_list[b / a.ncls] * a.T;  // this system's stage output
  bool bad = false;
  double2* win = swin + threadIdx.x;
  // ---- forward: positions j..j+kl in slots p mod W1 ----
  for (int p = 0; p <= kl && p < T; ++p) win[(p & (W1 - 1)) * S] = X[(size_t)p * 32];
  for (int j = 0; j < T - 1; ++j) {
    const int km = min(kl, T - 1 - j);
    double lv[KL];
#pragma unroll
    for (int i = 0; i < KL; ++i) lv[i] = (i < km) ? F[((size_t)j * ldab + kv + 1 + i) * 32] : 0.0;
    const int jp = P[(size_t)j * 32];
    const double2 inc = (j + kl + 1 < T) ? X[(size_t)(j + kl + 1) * 32] : zero2();
    const double2 bj = win[((j + jp) & (W1 - 1)) * S];
    if (jp) win[((j + jp) & (W1 - 1)) * S] = win[(j & (W1 - 1)) * S];
#pragma unroll
    for (int i = 0; i < KL; ++i) {
      if (i < km) {
        double2 w = win[((j + 1 + i) & (W1 - 1)) * S];
        w.x -= lv[i] * bj.x;
        w.y -= lv[i] * bj.y;
        win[((j + 1 + i) & (W1 - 1)) * S] = w;
      }
    }
    X[(size_t)j * 32] = bj;
    if (j + kl + 1 < T) win[((j + kl + 1) & (W1 - 1)) * S] = inc;
  }
  if (T > 0) X[(size_t)(T - 1) * 32] = win[((T - 1) & (W1 - 1)) * S];
  // ---- backward: x_{j+1}..x_{j+kv} in slots p mod W2 ----
  int sj = (T - 1) % W2;  // slot of position j
  for (int j = T - 1; j >= 0; --j) {
    const int im = min(kv, T - 1 - j);
    double u[KV];
#pragma unroll
    for (int i = 0; i < KV; ++i) u[i] = (i < im) ? F[((size_t)(j + 1 + i) * ldab + kv - 1 - i) * 32] : 0.0;
    const double dinv = F[((size_t)j * ldab + kv) * 32];  // U's diagonal is stored as its reciprocal
    double2 acc = X[(size_t)j * 32];
#pragma unroll
    for (int i = KV - 1; i >= 0; --i) {
      if (i < im) {
        int sl = sj + 1 + i;
        if (sl >= W2) sl -= W2;
        const double2 xv = win[sl * S];
        acc.x -= u[i] * xv.x;
        acc.y -= u[i] * xv.y;
      }
    }
    const double2 xj = make_double2(acc.x * dinv, acc.y * dinv);
    win[sj * S] = xj;
    {  // the solution, scaled back, straight into the stage output (original order)
      const int t = ccol[j];
      if (t >= 0) {
        const double2 xo = flip_col(xj, cflip[j]);
        bad |= !(isfinite(xo.x) && isfinite(xo.y));
        out[t] = xo;
      }
    }
    sj = (sj == 0) ? W2 - 1 : sj - 1;
  }
  if (bad) atomicOr(a.flags, 1u);
}

// ------------------------------------------------------------------------------
// Stage right-hand side with the NL assembly fused in, one CTA per (kx,ky) system
// (marching.f90:16-21, 93-125, 319-367):
//   Khat_i = sum_terms (i kx)^a (i ky)^b dsca trunc(I^Iz M^mz) qhat    (0 for inactive)
//   rhs    = M field + sum_{j<i} (dt a(i,j) Kstd_j + dt ahat(i+1,j) Khat_j) + dt ahat(i+1,i) Khat_i
// The system's quadratic-variable coefficients and state are first staged in
// shared memory with coalesced loads, so the row gathers run from shared memory.
// Active systems: rows flagged in rowflip are multiplied by -i for the real-scaled
// solve and the right-hand side goes to the solve's work layout.  Inactive systems
// (E = I): the right-hand side is the stage output itself (zero in the last
// stage), K_std_i = 0.
// ------------------------------------------------------------------------------
constexpr int kRhsThreads = 256;

__global__ void __launch_bounds__(kRhsThreads) k_rhs_nl(SolveArgs a, NLArgs n) {
  extern __shared__ double2 shr[];
  __shared__ double2 cms[kMaxGroups], cns[kMaxGroups];
  const int sid = blockIdx.x;
  const int T = a.T, NZ = a.d.NZ;
  const int kx = sid / a.d.NYA, ky = sid - kx * a.d.NYA;
  const int aidx = a.act_index[sid];
  const bool act = aidx >= 0;
  const bool origin = (kx == 0 && ky == 0);
  if (threadIdx.x < kMaxGroups) {
    const int g = threadIdx.x;
    cms[g] = (g < a.M.ngroups) ? cmul(ipow(a.kx[kx], a.M.gkx[g]), ipow(a.ky[ky], a.M.gky[g])) : zero2();
    cns[g] = (g < n.NL.ngroups) ? cmul(ipow(a.kx[kx], n.NL.gkx[g]), ipow(a.ky[ky], n.NL.gky[g])) : zero2();
  }
  const size_t base = (size_t)sid * T;
  const int nqz = act ? n.nq * NZ : 0;
  double2* qs = shr;         // [quad][n] of this (kx,ky)
  double2* fs = shr + nqz;   // state of this system
  {
    const size_t qstride = (size_t)a.d.NXH * a.d.NYA * NZ;  // between quad vars
    if (act) {
      // flat index idx = q NZ + nn, advanced without a division per element
      int q = threadIdx.x / NZ, nn = threadIdx.x - q * NZ;
      for (int idx = threadIdx.x; idx < nqz; idx += blockDim.x) {
        qs[idx] = n.qspec[q * qstride + (size_t)sid * NZ + nn];
        nn += blockDim.x;
        while (nn >= NZ) { nn -= NZ; ++q; }
      }
    }
    const double2* field = a.field + base;
    for (int t = threadIdx.x; t < T; t += blockDim.x) fs[t] = field[t];
  }
  __syncthreads();
  const bool zero_out = a.last_stage && !act;
  bool bad = false;
  for (int t = threadIdx.x; t < T; t += blockDim.x) {
    double2 kh = zero2();
    if (act) {
      // slots in batches of 4 independent loads; slots are filled in order and
      // exact zeros are not stored, so a zero ends the row
      for (int k0 = 0; k0 < n.NL.width; k0 += 4) {
        int cg[4];
        double v[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const bool ok = k0 + u < n.NL.width;
          cg[u] = ok ? n.NL.cg[(size_t)(k0 + u) * n.NL.rows + t] : 0;
          v[u] = ok ? n.NL.val[(size_t)(k0 + u) * n.NL.rows + t] : 0.0;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          if (v[u] != 0.0) {
            const double2 qh = qs[cg[u] & 0xFFFFFF];  // column = quad * NZ + n
            kh = cadd(kh, cmul(cns[cg[u] >> 24], make_double2(v[u] * qh.x, v[u] * qh.y)));
          }
        }
        if (v[3] == 0.0) break;
      }
    }
    // K_hat of the last stage is used only here, from the register (the next step
    // starts from K_hat_0)
    if (!a.last_stage) n.Khat[base + t] = kh;
    double2 r = zero2();
    if (!origin) {
#pragma unroll 4
      for (int k = 0; k < a.M.width; ++k) {
        const int cg = a.M.cg[(size_t)k * a.M.rows + t];
        const double v = a.M.val[(size_t)k * a.M.rows + t];
        const double2 xv = fs[cg & 0xFFFFFF];
        r = cadd(r, cmul(cms[cg >> 24], make_double2(v * xv.x, v * xv.y)));
      }
    }
#pragma unroll
    for (int j = 0; j < kMaxStages - 1; ++j) {  // static indices into the argument arrays
      if (j < a.nprev) {
        r = cadd(r, cscale(a.Kstd[j][base + t], a.ca[j]));
        r = cadd(r, cscale(a.Khat[j][base + t], a.ch[j]));
      }
    }
    r = cadd(r, cscale(kh, a.ch[a.nprev]));
    if (act) {
      if (a.rowflip) r = flip_row(r, a.rowflip[t]);
      if (a.work2) {  // thread-per-block layout, class order
        const int pos = a.row_pos[t], c = pos >= a.Tc ? 1 : 0, bb = aidx * a.ncls + c;
        a.work2[((size_t)(bb >> 5) * a.Tc + pos - c * a.Tc) * 32 + (bb & 31)] = r;
      } else {
        a.work[(size_t)sid * a.wst + (a.row_pos ? a.row_pos[t] : t)] = r;
      }
    } else {
      const double2 v = zero_out ? zero2() : r;
      bad |= !(isfinite(v.x) && isfinite(v.y));
      a.out[base + t] = v;
      if (a.Kstd_out) a.Kstd_out[base + t] = zero2();
    }
  }
  if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(a.flags, 1u);
}

// ------------------------------------------------------------------------------
// After the substitutions, one CTA per active system: the solution is staged in
// shared memory (from the solve's layout), then K_std_i = L x, the stage output
// (the new state in the last stage) and the non-finite check.
// ------------------------------------------------------------------------------
__global__ void __launch_bounds__(kRhsThreads) k_kstd_out(SolveArgs a) {
  extern __shared__ double2 xs[];
  __shared__ double2 cls[kMaxGroups];
  const int aidx = blockIdx.x;
  const int sid = a.act_list[aidx];
  const int T = a.T;
  const int kx = sid / a.d.NYA, ky = sid - kx * a.d.NYA;
  // thread-per-block solve: the solution is already in out, original order, and
  // only K_std remains (L with its original columns); whole-system solve: the
  // solution is in work (class order = original order), copied to out here
  const bool in_out = a.work2 != nullptr;
  const DevEll& L = in_out ? a.L : a.Lp;
  if (threadIdx.x < kMaxGroups) {
    const int g = threadIdx.x;
    cls[g] = (g < L.ngroups) ? cmul(ipow(a.kx[kx], L.gkx[g]), ipow(a.ky[ky], L.gky[g])) : zero2();
  }
  const size_t base = (size_t)sid * T;
  {
    const double2* x = in_out ? a.out + base : a.work + (size_t)sid * a.wst;
    for (int p = threadIdx.x; p < T; p += blockDim.x) xs[p] = x[p];
  }
  __syncthreads();
  bool bad = false;
  for (int t = threadIdx.x; t < T; t += blockDim.x) {
    if (!in_out) {
      const double2 v = xs[t];
      bad |= !(isfinite(v.x) && isfinite(v.y));
      if (a.out != a.work) a.out[base + t] = v;
    }
    if (a.Kstd_out) {
      double2 ks = zero2();
#pragma unroll 4
      for (int k = 0; k < L.width; ++k) {
        const int cg = L.cg[(size_t)k * L.rows + t];
        const double lv = L.val[(size_t)k * L.rows + t];
        const double2 xv = xs[cg & 0xFFFFFF];
        ks = cadd(ks, cmul(cls[cg >> 24], make_double2(lv * xv.x, lv * xv.y)));
      }
      a.Kstd_out[base + t] = ks;
    }
  }
  if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(a.flags, 1u);
}

// ------------------------------------------------------------------------------
// Operator-stationary K_std: a CTA takes one tile of kTileRows rows and kTileSys
// active systems.  Each thread keeps its row of L in grouped form (columns
// relative to the tile's solution window) in registers; the CTA first copies the
// windows of all its systems into shared memory (cp.async from the stage
// output), then evaluates its row for the systems one after the other: per
// monomial group a real sum, then one complex multiply by the group coefficient.
// ------------------------------------------------------------------------------
constexpr int kTileSys = 8;  // systems per CTA
constexpr int kLW = kGSlots;  // register slots of an L row (wider grouped L takes k_kstd_out)

// coefficient of group g of a grouped operator at (kx, ky)
__device__ __forceinline__ double2 gcoef(const DevGEll& G, int g, double kx, double ky) {
  double2 c = zero2();
  for (int m = 0; m < G.nmono[g]; ++m) c = cadd(c, cmul(ipow(kx, G.mkx[g][m]), ipow(ky, G.mky[g][m])));
  return c;
}
// one grouped row (slots in registers) applied to x: real sums per group, one
// complex multiply by the group coefficient c[g] per group
template <int RW>
__device__ __forceinline__ double2 grow(const DevGEll& G, const int* col, const double* val, const double2* x,
                                        const double2* c) {
  double2 r = zero2(), acc = zero2();
  int lg = 0;
#pragma unroll
  for (int k = 0; k < RW; ++k) {
    if (k < G.width) {
      if (k > 0 && G.slot_grp[k] != lg) {
        r = cadd(r, cmul(c[lg], acc));
        acc = zero2();
      }
      lg = G.slot_grp[k];
      if (val[k] != 0.0) {
        const double2 xv = x[col[k]];
        acc.x += val[k] * xv.x;
        acc.y += val[k] * xv.y;
      }
    }
  }
  if (G.width > 0) r = cadd(r, cmul(c[lg], acc));
  return r;
}

// G0..G3 > 0: the grouped L's slot ranges compiled (no run-time group test)
template <int G0 = 0, int G1 = 0, int G2 = 0, int G3 = 0>
__global__ void __launch_bounds__(kTileRows, 4) k_kstd_tiles(SolveArgs a) {
  extern __shared__ double2 xw[];
  __shared__ double2 cls[kTileSys][kMaxGroups];
  const int T = a.T;
  const int tile = blockIdx.x, t = tile * kTileRows + threadIdx.x;
  const bool row_ok = t < T;
  const int llo = a.tile_win[2 * tile], lw = a.tile_win[2 * tile + 1];
  const int a0 = blockIdx.y * kTileSys;
  const int ns = min(kTileSys, a.nact - a0);
  if (threadIdx.x < kTileSys * kMaxGroups) {
    const int u = threadIdx.x / kMaxGroups, g = threadIdx.x - u * kMaxGroups;
    const int sid = a.act_list[a0 + (u < ns ? u : 0)];
    const int kx = sid / a.d.NYA, ky = sid - kx * a.d.NYA;
    cls[u][g] = (g < a.Lw.ngroups) ? gcoef(a.Lw, g, a.kx[kx], a.ky[ky]) : zero2();
  }
  for (int u = 0; u < ns; ++u) {  // cp.async: no register round trip per system
    const double2* x = a.out + (size_t)a.act_list[a0 + u] * T + llo;
    for (int i = threadIdx.x; i < lw; i += kTileRows) cp_async16(xw + u * lw + i, x + i);
  }
  cp_async_commit();
  cp_async_wait<0>();
  __syncthreads();
  if (!row_ok) return;
  int lc[kLW];
  double lv[kLW];
#pragma unroll
  for (int k = 0; k < kLW; ++k) {
    const bool ok = k < a.Lw.width;
    lc[k] = ok ? a.Lw.col[k * a.Lw.rows + t] : 0;
    lv[k] = ok ? a.Lw.val[k * a.Lw.rows + t] : 0.0;
  }
  for (int u = 0; u < ns; ++u) {
    double2 ks;
    if constexpr (G0 > 0) {
      constexpr int W = G0 + G1 + G2 + G3;
      static_assert(W <= kLW, "grouped L slots");
      const double2* x = xw + u * lw;
      double2 acc[4] = {zero2(), zero2(), zero2(), zero2()};
#pragma unroll
      for (int k = 0; k < W; ++k) {
        const int g = k < G0 ? 0 : (k < G0 + G1 ? 1 : (k < G0 + G1 + G2 ? 2 : 3));
        if (lv[k] != 0.0) {
          const double2 xv = x[lc[k]];
          acc[g].x += lv[k] * xv.x;
          acc[g].y += lv[k] * xv.y;
        }
      }
      ks = cmul(cls[u][0], acc[0]);
      if (G1 > 0) ks = cadd(ks, cmul(cls[u][1], acc[1]));
      if (G2 > 0) ks = cadd(ks, cmul(cls[u][2], acc[2]));
      if (G3 > 0) ks = cadd(ks, cmul(cls[u][3], acc[3]));
    } else {
      ks = grow<kLW>(a.Lw, lc, lv, xw + u * lw, cls[u]);
    }
    a.Kstd_out[(size_t)a.act_list[a0 + u] * T + t] = ks;
  }
}

// ------------------------------------------------------------------------------
// Operator-stationary right-hand side: a CTA takes one tile of kTileRows rows
// and kRhsSys consecutive systems (active or not).  Each thread keeps its row of
// M and of the NL operator (columns relative to the tile's windows) in
// registers; the CTA copies the state window and the quadratic-variable windows
// of its systems into shared memory with cp.async, then evaluates its row: first
// K_hat and M x of every system from shared memory, then the earlier stages' K
// arrays (loads of all systems in flight together), then the stores.  Same
// arithmetic and order as k_rhs_nl.
// ------------------------------------------------------------------------------
constexpr int kRhsSys = 4;  // systems per CTA
constexpr int kRhsStg = 4;  // window entries per thread with precomputed offsets (wider: plain loops)

// G0, G1, G2 > 0: the NL operator in grouped form (SolveArgs::NLg) with slot
// ranges of these widths per monomial group, compiled: per group a real sum,
// then one complex multiply by the group coefficient (RN = G0 + G1 + G2)
template <int RM, int RN, int G0 = 0, int G1 = 0, int G2 = 0>
__global__ void __launch_bounds__(kTileRows, 6) k_rhs_tiles(SolveArgs a, NLArgs n) {
  extern __shared__ double2 win[];
  __shared__ double2 cms[kRhsSys][kMaxGroups], cns[kRhsSys][kMaxGroups];
  const int T = a.T, NZ = a.d.NZ, nsys = a.d.NXH * a.d.NYA;
  const int tile = blockIdx.y, t = tile * kTileRows + threadIdx.x;
  const int* rw = a.rhs_win + tile * kRhsWin;
  const int mlo = rw[0], mw = rw[1], nlo = rw[2], nw = rw[3], nqt = rw[4];
  const int ws = mw + nqt * nw;  // window entries per system
  const int s0 = blockIdx.x * kRhsSys, ns = min(kRhsSys, nsys - s0);
  const size_t qstride = (size_t)nsys * NZ;  // between quadratic variables of qspec
  if (ws <= kRhsStg * kTileRows) {
    // window entry e = threadIdx.x + j kTileRows: the same source offset for every
    // system (plus the system's base), computed once
    size_t off[kRhsStg];
#pragma unroll
    for (int j = 0; j < kRhsStg; ++j) {
      const int e = threadIdx.x + j * kTileRows;
      if (e < mw) {
        off[j] = (size_t)(mlo + e);
      } else {
        const int i = e - mw, sl = i / nw, k = i - sl * nw;
        off[j] = e < ws ? rw[5 + sl] * qstride + nlo + k : 0;
      }
    }
    for (int u = 0; u < ns; ++u) {
      const int sid = s0 + u;
      const bool act = a.act_index[sid] >= 0;
      double2* w = win + u * ws;
      const double2* f = a.field + (size_t)sid * T;
      const double2* qb = n.qspec + (size_t)sid * NZ;
#pragma unroll
      for (int j = 0; j < kRhsStg; ++j) {
        const int e = threadIdx.x + j * kTileRows;
        if (e < mw) cp_async16(w + e, f + off[j]);
        else if (e < ws && act) cp_async16(w + e, qb + off[j]);
      }
    }
  } else {
    for (int u = 0; u < ns; ++u) {
      const int sid = s0 + u;
      double2* w = win + u * ws;
      const double2* f = a.field + (size_t)sid * T + mlo;
      for (int i = threadIdx.x; i < mw; i += kTileRows) cp_async16(w + i, f + i);
      if (a.act_index[sid] >= 0)
        for (int i = threadIdx.x; i < nqt * nw; i += kTileRows) {
          const int sl = i / nw, k = i - sl * nw;
          cp_async16(w + mw + i, n.qspec + rw[5 + sl] * qstride + (size_t)sid * NZ + nlo + k);
        }
    }
  }
  cp_async_commit();
  for (int i = threadIdx.x; i < kRhsSys * kMaxGroups; i += kTileRows) {
    const int u = i / kMaxGroups, g = i - u * kMaxGroups;
    const int sid = s0 + (u < ns ? u : 0);
    const int kx = sid / a.d.NYA, ky = sid - kx * a.d.NYA;
    cms[u][g] = (g < a.Mw.ngroups) ? cmul(ipow(a.kx[kx], a.Mw.gkx[g]), ipow(a.ky[ky], a.Mw.gky[g])) : zero2();
    if constexpr (G0 > 0)
      cns[u][g] = (g < a.NLg.ngroups) ? gcoef(a.NLg, g, a.kx[kx], a.ky[ky]) : zero2();
    else
      cns[u][g] = (g < a.NLw.ngroups) ? cmul(ipow(a.kx[kx], a.NLw.gkx[g]), ipow(a.ky[ky], a.NLw.gky[g])) : zero2();
  }
  const bool row_ok = t < T;
  const int tr = row_ok ? t : 0;
  int mcg[RM], ncg[RN];
  double mv[RM], nv[RN];
#pragma unroll
  for (int k = 0; k < RM; ++k) {
    const bool ok = k < a.Mw.width;
    mcg[k] = ok ? a.Mw.cg[(size_t)k * a.Mw.rows + tr] : 0;
    mv[k] = ok ? a.Mw.val[(size_t)k * a.Mw.rows + tr] : 0.0;
  }
  constexpr bool kGrouped = G0 > 0;
  static_assert(!kGrouped || G0 + G1 + G2 == RN, "grouped NL slots");
#pragma unroll
  for (int k = 0; k < RN; ++k) {
    if constexpr (kGrouped) {
      ncg[k] = a.NLg.col[(size_t)k * a.NLg.rows + tr];
      nv[k] = a.NLg.val[(size_t)k * a.NLg.rows + tr];
    } else {
      const bool ok = k < a.NLw.width;
      ncg[k] = ok ? a.NLw.cg[(size_t)k * a.NLw.rows + tr] : 0;
      nv[k] = ok ? a.NLw.val[(size_t)k * a.NLw.rows + tr] : 0.0;
    }
  }
  // shared-memory index and group of every slot
  int nix[RN], ngr[RN], mix[RM], mgr[RM];
#pragma unroll
  for (int k = 0; k < RN; ++k) {
    nix[k] = mw + (ncg[k] & 0xFFFFFF);
    ngr[k] = kGrouped ? 0 : ncg[k] >> 24;
  }
#pragma unroll
  for (int k = 0; k < RM; ++k) {
    mix[k] = mcg[k] & 0xFFFFFF;
    mgr[k] = mcg[k] >> 24;
  }
  // M with the single monomial 1 (every recipe here): its coefficient is exactly
  // 1 and the complex multiply is skipped (identical for finite values)
  const bool m_unit = a.Mw.ngroups == 1 && a.Mw.gkx[0] == 0 && a.Mw.gky[0] == 0;
  int ai[kRhsSys];
#pragma unroll
  for (int u = 0; u < kRhsSys; ++u) ai[u] = u < ns ? a.act_index[s0 + u] : -1;
  cp_async_wait<0>();
  __syncthreads();
  if (!row_ok) return;  // no barrier below
  // phase 1 (shared memory only): K_hat and M x of every system
  double2 kh[kRhsSys], r[kRhsSys];
#pragma unroll
  for (int u = 0; u < kRhsSys; ++u) {
    kh[u] = zero2();
    r[u] = zero2();
    if (u < ns) {
      const double2* w = win + u * ws;
      if (ai[u] >= 0) {
        if constexpr (kGrouped) {
          double2 acc[3] = {zero2(), zero2(), zero2()};
#pragma unroll
          for (int k = 0; k < RN; ++k) {
            const int g = k < G0 ? 0 : (k < G0 + G1 ? 1 : 2);
            if (nv[k] != 0.0) {
              const double2 qh = w[nix[k]];
              acc[g].x += nv[k] * qh.x;
              acc[g].y += nv[k] * qh.y;
            }
          }
          kh[u] = cmul(cns[u][0], acc[0]);
          if (G1 > 0) kh[u] = cadd(kh[u], cmul(cns[u][1], acc[1]));
          if (G2 > 0) kh[u] = cadd(kh[u], cmul(cns[u][2], acc[2]));
        } else {
#pragma unroll
          for (int k = 0; k < RN; ++k)
            if (nv[k] != 0.0) {
              const double2 qh = w[nix[k]];
              kh[u] = cadd(kh[u], cmul(cns[u][ngr[k]], make_double2(nv[k] * qh.x, nv[k] * qh.y)));
            }
        }
      }
      if (s0 + u != 0) {
#pragma unroll
        for (int k = 0; k < RM; ++k)
          if (k < a.Mw.width) {
            const double2 xv = w[mix[k]];
            const double2 p = make_double2(mv[k] * xv.x, mv[k] * xv.y);
            r[u] = cadd(r[u], m_unit ? p : cmul(cms[u][mgr[k]], p));
          }
      }
    }
  }
  // phase 2: the earlier stages' K arrays (no store in between: the loads of all
  // systems can be in flight together)
#pragma unroll
  for (int j = 0; j < kMaxStages - 1; ++j) {  // static indices into the argument arrays
    if (j < a.nprev) {
#pragma unroll
      for (int u = 0; u < kRhsSys; ++u)
        if (u < ns) {
          const size_t base = (size_t)(s0 + u) * T + t;
          r[u] = cadd(r[u], cscale(a.Kstd[j][base], a.ca[j]));
          r[u] = cadd(r[u], cscale(a.Khat[j][base], a.ch[j]));
        }
    }
  }
  // phase 3: stores
  const int pos = a.row_pos[t], c = pos >= a.Tc ? 1 : 0, pc = pos - c * a.Tc;
  const unsigned char rf = a.rowflip ? a.rowflip[t] : 0;
  bool bad = false;
#pragma unroll
  for (int u = 0; u < kRhsSys; ++u) {
    if (u >= ns) break;
    const size_t base = (size_t)(s0 + u) * T;
    // K_hat of the last stage is used only here, from the register
    if (!a.last_stage) n.Khat[base + t] = kh[u];
    double2 v = cadd(r[u], cscale(kh[u], a.ch[a.nprev]));
    if (ai[u] >= 0) {
      if (a.rowflip) v = flip_row(v, rf);
      const int bb = ai[u] * a.ncls + c;
      a.work2[((size_t)(bb >> 5) * a.Tc + pc) * 32 + (bb & 31)] = v;
    } else {
      if (a.last_stage) v = zero2();
      bad |= !(isfinite(v.x) && isfinite(v.y));
      a.out[base + t] = v;
      if (a.Kstd_out) a.Kstd_out[base + t] = zero2();
    }
  }
  if (bad) atomicOr(a.flags, 1u);
}

// ------------------------------------------------------------------------------
// mean (kx = ky = 0) systems: real arithmetic, one warp per system
// ------------------------------------------------------------------------------
__device__ double ell_row_real(const DevEll& op, int t, const double* x) {
  double acc = 0.0;
  for (int k = 0; k < op.width; ++k) acc += op.v(t, k) * x[op.col(t, k)];
  return acc;
}

__global__ void k_zero_step(ZeroArgs a) {
  extern __shared__ double smd[];
  const int lane = threadIdx.x;
  const int s = blockIdx.x;
  if (s >= a.nsys) return;
  const ZeroSysDev& z = a.sys[s];
  const int T = z.T, i = a.stage;
  double* b = smd;
  double* kh = a.sys[s].Khat[i];
  // NL: K_hat_i from the real part of the (0,0) Chebyshev coefficients (marching.f90:372-397)
  for (int t = lane; t < T; t += 32) {
    double acc = 0.0;
    for (int k = 0; k < z.NL.width; ++k) {
      const int c = z.NL.col(t, k);
      const int qv = c / a.d.NZ, n = c - qv * a.d.NZ;
      acc += z.NL.v(t, k) * a.qspec[(size_t)qv * a.d.NXH * a.d.NYA * a.d.NZ + n].x;
    }
    if (z.src) acc += z.src[t];
    kh[t] = acc;
  }
  __syncwarp();
  for (int t = lane; t < T; t += 32) {
    double r = ell_row_real(z.M, t, z.field);
    for (int j = 0; j < i; ++j) {
      r = r + a.ca[j] * z.Kstd[j][t];
      r = r + a.ch[j] * z.Khat[j][t];
    }
    r = r + a.ch[i] * kh[t];
    b[t] = r;
  }
  // band solve with the factors staged in shared memory; the updates of one
  // column run across the lanes (each entry sees the same sequence of updates)
  const int kl = z.kl, kv = z.kl + z.ku, ldab = z.ldab;
  double* fab = smd + T;
  for (int e = lane; e < T * ldab; e += 32) fab[e] = z.ab[e];
  __syncwarp();
  for (int j = 0; j < T - 1; ++j) {
    const int p = j + z.dpiv[j];
    if (lane == 0 && p != j) { const double tmp = b[p]; b[p] = b[j]; b[j] = tmp; }
    __syncwarp();
    const double bj = b[j];
    const int lm = min(kl, T - 1 - j);
    for (int q = 1 + lane; q <= lm; q += 32) b[j + q] -= fab[j * ldab + kv + q] * bj;
    __syncwarp();
  }
  for (int j = T - 1; j >= 0; --j) {
    const double bj = b[j] * fab[j * ldab + kv];
    __syncwarp();
    if (lane == 0) b[j] = bj;
    for (int q = 1 + lane; q <= kv && j - q >= 0; q += 32) b[j - q] -= fab[j * ldab + kv - q] * bj;
    __syncwarp();
  }
  double* out = a.last_stage ? z.field : z.aux;
  if (!a.last_stage)
    for (int t = lane; t < T; t += 32) z.Kstd[i][t] = ell_row_real(z.L, t, b);
  __syncwarp();
  for (int t = lane; t < T; t += 32) out[t] = b[t];
}

__global__ void k_zero_factor(ZeroArgs a) {
  const int s = blockIdx.x;
  if (s >= a.nsys || threadIdx.x != 0) return;
  const ZeroSysDev& z = a.sys[s];
  const int T = z.T, kl = z.kl, ku = z.ku, kv = kl + ku, ldab = z.ldab;
  double* ab = z.ab;
  for (size_t e = 0; e < (size_t)T * ldab; ++e) ab[e] = 0.0;
  for (int t = 0; t < T; ++t) {
    for (int k = 0; k < z.M.width; ++k) {
      const double v = z.M.v(t, k);
      if (v == 0.0) continue;
      const int c = z.M.col(t, k);
      ab[(size_t)c * ldab + kv + t - c] += v;
    }
    for (int k = 0; k < z.L.width; ++k) {
      const double v = z.L.v(t, k);
      if (v == 0.0) continue;
      const int c = z.L.col(t, k);
      ab[(size_t)c * ldab + kv + t - c] += a.zsca * v;
    }
  }
  int ju = 0, info = 0;
  for (int j = 0; j < T; ++j) {
    const int km = min(kl, T - 1 - j);
    int jp = 0;
    double best = -1.0;
    for (int q = 0; q <= km; ++q) {
      const double v = fabs(ab[(size_t)j * ldab + kv + q]);
      if (v > best) { best = v; jp = q; }
    }
    z.dpiv[j] = (unsigned char)jp;
    if (ab[(size_t)j * ldab + kv + jp] == 0.0) { if (!info) info = j + 1; continue; }
    ju = max(ju, min(j + ku + jp, T - 1));
    if (jp != 0)
      for (int c = j; c <= ju; ++c) {
        double* p1 = ab + (size_t)c * ldab + kv + j + jp - c;
        double* p0 = ab + (size_t)c * ldab + kv + j - c;
        double t0 = *p0; *p0 = *p1; *p1 = t0;
      }
    const double r = 1.0 / ab[(size_t)j * ldab + kv];
    for (int q = 1; q <= km; ++q) ab[(size_t)j * ldab + kv + q] *= r;
    for (int c = j + 1; c <= ju; ++c) {
      const double rowv = ab[(size_t)c * ldab + kv + j - c];
      for (int q = 1; q <= km; ++q) ab[(size_t)c * ldab + kv + j + q - c] -= ab[(size_t)j * ldab + kv + q] * rowv;
    }
    ab[(size_t)j * ldab + kv] = r;
  }
  a.info[s] = info;
}

// ------------------------------------------------------------------------------
// QuickSave / checkpoint helpers
// ------------------------------------------------------------------------------
__global__ void k_transpose_xy(Dims d, const double* in, double* out, int to_file) {
  const size_t n = (size_t)d.NXA * d.NYA * d.NZA;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    const int z = (int)(e % d.NZA);
    const size_t r = e / d.NZA;
    // e indexes the output array
    if (to_file) {  // out[x][y][z] <- in[y][x][z]
      const int y = (int)(r % d.NYA), x = (int)(r / d.NYA);
      out[e] = in[((size_t)y * d.NXA + x) * d.NZA + z];
    } else {        // out[y][x][z] <- in[x][y][z]
      const int x = (int)(r % d.NXA), y = (int)(r / d.NXA);
      out[e] = in[((size_t)x * d.NYA + y) * d.NZA + z];
    }
  }
}

// ------------------------------------------------------------------------------
// User outputs (coral.usrOutput, PL_equations.f90:322-427) of one physical field
// phys[y][x][z], in the reference's file order (transforms.f90:53-105,772-866):
//   kind 1 ZSlice at z index k:  out[x][y] = phys(z = k)
//   kind 2 YSlice at y index k:  out[x][z] = phys(y = k)
//   kind 3 XSlice at x index k:  out[y][z] = phys(x = k)
//   kind 4 Zsummed:              out[x][y] = sum_z w(z) phys, z in grid order
// (indices 0-based here).  Profiles: k_usr_profile.
// ------------------------------------------------------------------------------
__global__ void k_usr_slice(Dims d, const double* phys, int kind, int k, const double* wz, double* out) {
  const size_t n = kind == 1 || kind == 4 ? (size_t)d.NXA * d.NYA
                   : kind == 2          ? (size_t)d.NXA * d.NZA
                                        : (size_t)d.NYA * d.NZA;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    double v;
    if (kind == 1 || kind == 4) {
      const int y = (int)(e % d.NYA), x = (int)(e / d.NYA);
      const double* col = phys + ((size_t)y * d.NXA + x) * d.NZA;
      if (kind == 1) {
        v = col[k];
      } else {
        v = 0.0;
        for (int z = 0; z < d.NZA; ++z) v += col[z] * wz[z];
      }
    } else if (kind == 2) {
      const int z = (int)(e % d.NZA), x = (int)(e / d.NZA);
      v = phys[((size_t)k * d.NXA + x) * d.NZA + z];
    } else {
      const int z = (int)(e % d.NZA), y = (int)(e / d.NZA);
      v = phys[((size_t)y * d.NXA + k) * d.NZA + z];
    }
    out[e] = v;
  }
}

// Horizontal average profile (export_Profile_fftw_mpi, PL_IMEX_timestepping_output.f90:
// 489-581): one CTA per z level, sum over x and y, then / NXAA / NYAA.
__global__ void __launch_bounds__(256) k_usr_profile(Dims d, const double* phys, double* out) {
  __shared__ double red[8];
  const int z = blockIdx.x;
  double s = 0.0;
  for (size_t e = threadIdx.x; e < (size_t)d.NXA * d.NYA; e += blockDim.x) s += phys[e * d.NZA + z];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < 8; ++w) t += red[w];
    out[z] = t / d.NXA / d.NYA;
  }
}

// product of two physical fields (a quadratic variable), or a copy when b is null
__global__ void k_phys_product(size_t n, const double* a, const double* b, double* out) {
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x)
    out[e] = b ? a[e] * b[e] : a[e];
}

// ------------------------------------------------------------------------------
// z derivatives in full-variable builds (compute_full_variables_in_physical_space,
// marching.f90:455-466, with differentiate_kxky, PL_IMEX_timestepping.f90:276-319):
// per (kx, ky) column, the Chebyshev coefficients of one kxky variable (its
// Galerkin stencil applied to the state) times dsca, differentiated `order`
// times -- the coefficients shifted down by one and back-substituted against
// the Chebyshev integration operator trunc(I)[rows 2..NZ, cols 1..NZ-1] (upper
// triangular: diagonal gap/2 at n = 0, gap/(4(n+1)) beyond; second
// super-diagonal -gap/(4(n+1)); prepare_chebyshev_integration, :488-505), the
// last coefficient zero -- into out[kx][ky][n].  One thread per column; the
// back substitution runs in place with the values it still needs in registers.
// ------------------------------------------------------------------------------
__global__ void k_full_dz(Dims d, const double2* state, int T, const int* tab_t, const double* tab_v, double dsca,
                          int order, double gap, double2* out) {
  const size_t ncol = (size_t)d.NXH * d.NYA;
  const int NZ = d.NZ;
  for (size_t col = (size_t)blockIdx.x * blockDim.x + threadIdx.x; col < ncol; col += (size_t)gridDim.x * blockDim.x) {
    const double2* sv = state + col * T;
    double2* o = out + col * NZ;
    for (int n = 0; n < NZ; ++n) {
      double2 c = zero2();
      for (int k = 0; k < kTabW; ++k) {
        const int tt = tab_t[n * kTabW + k];
        if (tt >= 0) {
          const double w = tab_v[n * kTabW + k];
          const double2 x = sv[tt];
          c.x += w * x.x;
          c.y += w * x.y;
        }
      }
      o[n] = cscale(c, dsca);
    }
    for (int r = 0; r < order; ++r) {
      double2 chi = o[NZ - 1];                 // c(n + 1), not yet overwritten
      double2 dp1 = zero2(), dp2 = zero2();    // d(n + 1), d(n + 2)
      for (int n = NZ - 2; n >= 0; --n) {
        const double2 cn = o[n];
        const double diag = (n == 0) ? 0.5 * gap : gap / (4.0 * (n + 1));
        const double sup = -gap / (4.0 * (n + 1));
        const double2 v = (n + 2 <= NZ - 2) ? make_double2(chi.x - sup * dp2.x, chi.y - sup * dp2.y) : chi;
        const double2 dn = make_double2(v.x / diag, v.y / diag);
        o[n] = dn;
        chi = cn;
        dp2 = dp1;
        dp1 = dn;
      }
      o[NZ - 1] = zero2();
    }
  }
}

// The same for a mean variable (differentiate_zero, PL_IMEX_timestepping.f90:
// 321-360): one real profile, one thread.
__global__ void k_zero_dz(int NZ, const double* state, const int* tab_t, const double* tab_v, double dsca,
                          int order, double gap, double* out) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  for (int n = 0; n < NZ; ++n) {
    double c = 0.0;
    for (int k = 0; k < kTabW; ++k) {
      const int tt = tab_t[n * kTabW + k];
      if (tt >= 0) c += tab_v[n * kTabW + k] * state[tt];
    }
    out[n] = c * dsca;
  }
  for (int r = 0; r < order; ++r) {
    double chi = out[NZ - 1], dp1 = 0.0, dp2 = 0.0;
    for (int n = NZ - 2; n >= 0; --n) {
      const double cn = out[n];
      const double diag = (n == 0) ? 0.5 * gap : gap / (4.0 * (n + 1));
      const double sup = -gap / (4.0 * (n + 1));
      const double v = (n + 2 <= NZ - 2) ? chi - sup * dp2 : chi;
      const double dn = v / diag;
      out[n] = dn;
      chi = cn;
      dp2 = dp1;
      dp1 = dn;
    }
    out[NZ - 1] = 0.0;
  }
}

// Projection of Chebyshev coefficients onto one variable's Galerkin basis
// (square-stencil solve of import_quicksave, PL_IMEX_timestepping_output.f90:343-355).
// The square stencil is lower triangular, so a forward substitution solves it;
// the caller has zeroed the state, so the result is written into the slots.
__global__ void k_galerkin_insert(Dims d, const double2* spec, int T, const int* var_pos, int nc,
                                  const double* sq, const int* sq_col, double2* field) {
  const size_t col = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= (size_t)d.NXH * d.NYA) return;
  const double2* c = spec + col * d.NZ;
  double2* f = field + col * T;
  for (int r = 0; r < nc; ++r) {
    double2 acc = c[r];
    double diag = 1.0;
    for (int k = 0; k < kTabW; ++k) {
      const int cc = sq_col[r * kTabW + k];
      if (cc < 0) continue;
      const double v = sq[r * kTabW + k];
      if (cc == r) diag = v;
      else if (cc < r) acc = csub(acc, cscale(f[var_pos[cc]], v));
    }
    f[var_pos[r]] = make_double2(acc.x / diag, acc.y / diag);
  }
}

__global__ void k_cheb_extract(Dims d, const double2* field, int T, const int* tab_t, const double* tab_v,
                               double2* spec) {
  const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t n_all = (size_t)d.NXH * d.NYA * d.NZ;
  if (e >= n_all) return;
  const int n = (int)(e % d.NZ);
  const size_t col = e / d.NZ;
  const double2* f = field + col * T;
  double2 s = zero2();
  for (int k = 0; k < kTabW; ++k) {
    const int tt = tab_t[n * kTabW + k];
    if (tt >= 0) s = cadd(s, cscale(f[tt], tab_v[n * kTabW + k]));
  }
  spec[e] = s;
}

__global__ void k_check_finite(const double2* x, size_t n, unsigned int* flags) {
  bool bad = false;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x)
    bad |= !(isfinite(x[e].x) && isfinite(x[e].y));
  if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(flags, 1u);
}

int grid1d(size_t n, int bs) { return (int)((n + bs - 1) / bs); }

// Raise a kernel's dynamic shared-memory limit when its static plus dynamic
// shared memory exceeds the default 48 KB (a launch above it without the
// attribute is an invalid argument); a refused attribute is reported with the
// kernel and the size (instead of surfacing later as a generic launch failure).
template <typename K>
void set_smem_named(const char* name, K kernel, size_t bytes) {
  size_t stat = 0;
  cudaFuncAttributes fa;
  if (cudaFuncGetAttributes(&fa, kernel) == cudaSuccess) stat = fa.sharedSizeBytes;
  else cudaGetLastError();
  if (bytes + stat <= 48 * 1024) return;
  const cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();  // the refusal is reported here, not left for the next launch check
    throw CoralError(CORAL_ECUDA, std::string("cudaFuncSetAttribute(") + name + ", dynamic shared memory " +
                                      std::to_string(bytes) + " bytes): " + cudaGetErrorString(e));
  }
}
// (variadic so that template argument lists pass through; the text names the call)
#define set_smem(...) set_smem_named(#__VA_ARGS__, __VA_ARGS__)

}  // namespace

// ---- launchers ----------------------------------------------------------------
// Each transform kernel is instantiated for the lengths of the usual grids
// (compile-time FFT plans); other lengths use the runtime plan.
#define CORAL_FFT_LENGTHS(X) X(24) X(36) X(48) X(72) X(96) X(144) X(192) X(288) X(384) X(576)

template <template <int> class L, typename... Args>
void dispatch_len(int n, Args&&... args) {
  switch (n) {
#define CORAL_CASE(v) \
  case v:             \
    L<v>::run(args...); \
    return;
    CORAL_FFT_LENGTHS(CORAL_CASE)
#undef CORAL_CASE
    default:
      L<0>::run(args...);
  }
}

// CTAs of a persistent kernel: as many as fit on the device at once
template <class K>
int persistent_ctas(K kernel, int threads, size_t smem) {
  int dev = 0, nsm = 0, per = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, threads, smem);
  return std::max(1, nsm * std::max(per, 1));
}

template <int NF>
struct InvY {
  static void run(const Dims& d, int nf, const FullVarDev* fv, StateSet st, const double2* plain_spec,
                  const double* kx, const double* ky, double2* Y1, const FftPlan& py, int single, cudaStream_t s) {
    size_t sm = (NF ? 1 : 2) * kNB1 * (size_t)(d.NYA + kPadY) * sizeof(double2);
    dim3 g(nf, (d.NZ + kNB1 - 1) / kNB1, d.NXH);
    if (single && !plain_spec) {
      set_smem(k_inv_y1<NF>, sm);
      k_inv_y1<NF><<<g, kThreadsY, sm, s>>>(d, fv, st, kx, ky, Y1, py);
      return;
    }
    set_smem(k_inv_y<NF>, sm);
    k_inv_y<NF><<<g, kThreadsY, sm, s>>>(d, fv, st, plain_spec, kx, ky, Y1, py);
  }
};
template <int NF>
struct InvX {
  template <int PV>
  static void go(const Dims& d, int nf, const double2* Y1, double* Y2, const FftPlan& px, cudaStream_t s) {
    go<PV>(d, nf, Y1, Y2, px, 0, d.NYA, s);
  }
  template <int PV>
  static void go(const Dims& d, int nf, const double2* Y1, double* Y2, const FftPlan& px, int y0, int ny,
                 cudaStream_t s) {
    size_t sm = (NF ? 1 : 2) * (kNB2 / 2) * (size_t)(d.NXA + kPadXY) * sizeof(double2);
    set_smem(k_inv_x<NF, PV>, sm);
    dim3 g(nf, (d.NZ + kNB2 - 1) / kNB2, ny);
    k_inv_x<NF, PV><<<g, kThreadsX, sm, s>>>(d, Y1, Y2, px, y0);
  }
  static void rows(const Dims& d, int nf, const double2* Y1, double* Y2, const FftPlan& px, int pv, int y0, int ny,
                   cudaStream_t s) {
    if (pv) go<1>(d, nf, Y1, Y2, px, y0, ny, s);
    else go<0>(d, nf, Y1, Y2, px, y0, ny, s);
  }
  static void run(const Dims& d, int nf, const double2* Y1, double* Y2, const FftPlan& px, int pv, int tiles,
                  cudaStream_t s) {
    if constexpr (NF != 0 && tw_pass2_len<NF, 1>() > 0) {
      if (pv && !tiles) {
        // persistent pipelined kernel: as many CTAs as fit on the device at once
        const size_t sm = ((kNB2 / 2) * (size_t)(NF + kPadXY) + (size_t)d.NXH * kStgX) * sizeof(double2);
        set_smem(k_inv_x_pipe<NF>, sm);
        static int nct = 0;
        if (!nct) nct = persistent_ctas(k_inv_x_pipe<NF>, kThreadsXP, sm);
        const int ntiles = nf * ((d.NZ + kNB2 - 1) / kNB2) * d.NYA;
        k_inv_x_pipe<NF><<<std::min(nct, ntiles), kThreadsXP, sm, s>>>(d, nf, Y1, Y2, px);
        return;
      }
    }
    if (pv) go<1>(d, nf, Y1, Y2, px, s);
    else go<0>(d, nf, Y1, Y2, px, s);
  }
};
template <int NF>
struct InvZ {
  static void run(const Dims& d, int nf, const double* Y2, double* phys, const FftPlan& pz, const double2* dct_tw,
                  const double* wz, unsigned long long* cfl_bits, cudaStream_t s) {
    size_t sm = (NF ? 1 : 2) * (kXB3 / 2) * (size_t)d.NZA * sizeof(double2);
    set_smem(k_inv_z<NF>, sm);
    dim3 g(nf, (d.NXA + kXB3 - 1) / kXB3, d.NYA);
    k_inv_z<NF><<<g, kThreads, sm, s>>>(d, Y2, phys, pz, dct_tw, wz, cfl_bits);
  }
};
template <int NF>
struct FwdZ {
  static void run(const Dims& d, int nf, const QuadDesc& q, const double* phys, double* Q2, const FftPlan& pz,
                  const double2* dct_tw, const double* wz, double* ke_partial, cudaStream_t s) {
    size_t sm = (size_t)nf * d.NZA * sizeof(double2) + (NF ? 1 : 2) * (size_t)std::min(q.nq, kQC) * d.NZA * sizeof(double2);
    set_smem(k_fwd_z<NF>, sm);
    dim3 g((d.NXA + 1) / 2, d.NYA);
    k_fwd_z<NF><<<g, kThreads, sm, s>>>(d, nf, q, phys, Q2, pz, dct_tw, wz, ke_partial);
  }
};
template <int NF>
struct ZFused {
  template <int FB>
  static void go(const Dims& d, int nf, const QuadDesc& q, const double* Y2, double* Q2, const FftPlan& pz,
                 const double2* dct_tw, const double* wz, const double* wzinv, unsigned long long* cfl_bits,
                 double* ke_partial, int y0, int ny, cudaStream_t s) {
    const size_t lines = (size_t)nf * kZPairs + FB + (NF ? 0 : std::max(kZLines, FB));
    const size_t sm = lines * d.NZA * sizeof(double2);
    set_smem(k_z_fused<NF, FB>, sm);
    dim3 g((d.NXA + 2 * kZPairs - 1) / (2 * kZPairs), ny);
    k_z_fused<NF, FB><<<g, z_threads_fused(NF, FB), sm, s>>>(d, nf, q, Y2, Q2, pz, dct_tw, wz, wzinv, cfl_bits,
                                                               ke_partial, y0);
  }
  static void run(const Dims& d, int nf, const QuadDesc& q, const double* Y2, double* Q2, const FftPlan& pz,
                  const double2* dct_tw, const double* wz, const double* wzinv, unsigned long long* cfl_bits,
                  double* ke_partial, int batch6, int y0, int ny, cudaStream_t s) {
    if (NF != 0 && 3 * d.NZ != 2 * NF) {  // compiled lengths assume NZAA = 3 NZ / 2
      ZFused<0>::run(d, nf, q, Y2, Q2, pz, dct_tw, wz, wzinv, cfl_bits, ke_partial, batch6, y0, ny, s);
      return;
    }
    if (batch6 && nf <= 4) go<6>(d, nf, q, Y2, Q2, pz, dct_tw, wz, wzinv, cfl_bits, ke_partial, y0, ny, s);
    else go<kZFwd>(d, nf, q, Y2, Q2, pz, dct_tw, wz, wzinv, cfl_bits, ke_partial, y0, ny, s);
  }
};
template <int NF>
struct FwdX {
  template <int PV>
  static void go(const Dims& d, int nq, const double* Q2, double2* Q1, const FftPlan& px, int y0, int ny,
                 cudaStream_t s) {
    size_t sm = (NF ? 1 : 2) * (kNB2 / 2) * (size_t)(d.NXA + kPadXY) * sizeof(double2);
    set_smem(k_fwd_x<NF, PV>, sm);
    dim3 g(nq, (d.NZ + kNB2 - 1) / kNB2, ny);
    k_fwd_x<NF, PV><<<g, kThreadsX, sm, s>>>(d, Q2, Q1, px, y0);
  }
  static void run(const Dims& d, int nq, const double* Q2, double2* Q1, const FftPlan& px, int pv, int y0, int ny,
                  cudaStream_t s) {
    if (pv) go<1>(d, nq, Q2, Q1, px, y0, ny, s);
    else go<0>(d, nq, Q2, Q1, px, y0, ny, s);
  }
};
template <int NF>
struct FwdY {
  static void run(const Dims& d, int nq, const double2* Q1, double2* qspec, double scale, const FftPlan& py,
                  int grid_variant, cudaStream_t s) {
    if constexpr (NF != 0) {
      if (!grid_variant) {
      // persistent pipelined kernel: as many CTAs as fit on the device at once
      const size_t sm = (kNB1 * (size_t)(NF + kPadY) + (size_t)NF * kNB1) * sizeof(double2);
      set_smem(k_fwd_y_pipe<NF>, sm);
      static int nct = 0;
      if (!nct) nct = persistent_ctas(k_fwd_y_pipe<NF>, kThreadsYF, sm);
      const int ntiles = nq * ((d.NZ + kNB1 - 1) / kNB1) * d.NXH;
      k_fwd_y_pipe<NF><<<std::min(nct, ntiles), kThreadsYF, sm, s>>>(d, nq, Q1, qspec, scale, py);
      return;
    }
    }
    size_t sm = (NF ? 1 : 2) * kNB1 * (size_t)(d.NYA + kPadY) * sizeof(double2);
    set_smem(k_fwd_y<NF>, sm);
    dim3 g(nq, (d.NZ + kNB1 - 1) / kNB1, d.NXH);
    k_fwd_y<NF><<<g, kThreadsY, sm, s>>>(d, Q1, qspec, scale, py);
  }
};

void launch_inv_y(const Dims& d, int nf, const FullVarDev* fv, StateSet st, const double2* plain_spec,
                  const double* kx, const double* ky, double2* Y1, const FftPlan& py, cudaStream_t s, int single) {
  dispatch_len<InvY>(d.NYA, d, nf, fv, st, plain_spec, kx, ky, Y1, py, single, s);
}
void launch_z_fused(const Dims& d, int nf, const QuadDesc& q, const double* Y2, double* Q2, const FftPlan& pz,
                    const double2* dct_tw, const double* wz, const double* wzinv, unsigned long long* cfl_bits,
                    double* ke_partial, cudaStream_t s, int batch6, int y0, int ny) {
  if (ny < 0) ny = d.NYA - y0;
  dispatch_len<ZFused>(d.NZA, d, nf, q, Y2, Q2, pz, dct_tw, wz, wzinv, cfl_bits, ke_partial, batch6, y0, ny, s);
}
template <int NF>
struct InvXRows {
  static void run(const Dims& d, int nf, const double2* Y1, double* Y2, const FftPlan& px, int pv, int y0, int ny,
                  cudaStream_t s) {
    InvX<NF>::rows(d, nf, Y1, Y2, px, pv, y0, ny, s);
  }
};
void launch_inv_x_rows(const Dims& d, int nf, const double2* Y1, double* Y2, const FftPlan& px, int pv, int y0, int ny,
                       cudaStream_t s) {
  dispatch_len<InvXRows>(d.NXA, d, nf, Y1, Y2, px, pv, y0, ny, s);
}
void launch_inv_x(const Dims& d, int nf, const double2* Y1, double* Y2, const FftPlan& px, cudaStream_t s, int pv,
                  int tiles) {
  dispatch_len<InvX>(d.NXA, d, nf, Y1, Y2, px, pv, tiles, s);
}
void launch_inv_z(const Dims& d, int nf, const double* Y2, double* phys, const FftPlan& pz,
                  const double2* dct_tw, const double* wz, unsigned long long* cfl_bits, cudaStream_t s) {
  dispatch_len<InvZ>(d.NZA, d, nf, Y2, phys, pz, dct_tw, wz, cfl_bits, s);
}
void launch_fwd_z(const Dims& d, int nf, const QuadDesc& q, const double* phys, double* Q2, const FftPlan& pz,
                  const double2* dct_tw, const double* wz, double* ke_partial, cudaStream_t s) {
  dispatch_len<FwdZ>(d.NZA, d, nf, q, phys, Q2, pz, dct_tw, wz, ke_partial, s);
}
void launch_fwd_x(const Dims& d, int nq, const double* Q2, double2* Q1, const FftPlan& px, cudaStream_t s, int pv,
                  int y0, int ny) {
  if (ny < 0) ny = d.NYA - y0;
  dispatch_len<FwdX>(d.NXA, d, nq, Q2, Q1, px, pv, y0, ny, s);
}
void launch_fwd_y(const Dims& d, int nq, const double2* Q1, double2* qspec, double scale, const FftPlan& py,
                  cudaStream_t s, int grid_variant) {
  dispatch_len<FwdY>(d.NYA, d, nq, Q1, qspec, scale, py, grid_variant, s);
}
// total of the KE partial sums written by the z kernels: one CTA, each thread a
// strided sum, then a fixed-order tree
__global__ void __launch_bounds__(1024) k_ke_sum(const double* part, size_t n, double* out) {
  __shared__ double red[32];
  double v = 0.0;
  for (size_t i = threadIdx.x; i < n; i += blockDim.x) v += part[i];
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x < 32) {
    v = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (threadIdx.x == 0) *out = v;
  }
}
size_t z_fused_ctas(const Dims& d) { return (size_t)((d.NXA + 2 * kZPairs - 1) / (2 * kZPairs)) * d.NYA; }
void launch_ke_sum(const double* part, size_t n, double* out, cudaStream_t s) {
  k_ke_sum<<<1, 1024, 0, s>>>(part, n, out);
}
void launch_remove_zmean(const Dims& d, double2* qspec_q, cudaStream_t s) {
  k_remove_zmean<<<grid1d((size_t)d.NXH * d.NYA, 128), 128, 0, s>>>(d, qspec_q);
}

// ------------------------------------------------------------------------------
// full variables that are not plain transforms (marching.f90:505-575)
// ------------------------------------------------------------------------------
namespace {

// z operations of one CTA on kZfCols consecutive x columns of one y row, whose
// Chebyshev coefficients are contiguous in Y2: the tile is staged in shared
// memory and each column runs the reference's loops in its order.  Y2 holds
// c_0 and c_n / 2 (n >= 1; the inverse y pass folds the x padding's 0.5 and
// the REDFT01 convention in), so every c_n (n >= 1) read into c_0 is 2 Y2[n]
// (exact).
constexpr int kZfCols = 16;
__global__ void k_zfilter(Dims d, double* Y2v, int extract, int decomp, int y0) {
  extern __shared__ double tile[];
  const int NZ = d.NZ, y = y0 + blockIdx.y, xc0 = blockIdx.x * kZfCols;
  const int nc = min(kZfCols, d.NXA - xc0);
  double* base = Y2v + ((size_t)y * d.NXA + xc0) * NZ;
  for (int i = threadIdx.x; i < nc * NZ; i += blockDim.x) tile[i] = base[i];
  __syncthreads();
  if ((int)threadIdx.x < nc) {
    double* c = tile + threadIdx.x * NZ;
    if (extract == 1) {  // bottom surface: T_n(-1) = (-1)^n
      for (int iz = 2; iz <= NZ; ++iz) {
        c[0] = c[0] - (2.0 * c[iz - 1]) * ((iz & 1) ? -1.0 : 1.0);
        c[iz - 1] = 0.0;
      }
    } else if (extract == 2) {  // top surface: T_n(1) = 1
      for (int iz = 2; iz <= NZ; ++iz) {
        c[0] = c[0] + 2.0 * c[iz - 1];
        c[iz - 1] = 0.0;
      }
    }
    if (decomp == 2) {  // baroclinic: the vertical mean removed (PL_IMEX_timestepping.f90:238-250)
      c[0] = 0.0;
      for (int q = 1; q < NZ / 2; ++q)
        c[0] = c[0] - (2.0 * c[2 * q]) * (0.5 / (2.0 * q + 1.0) - 0.5 / (2.0 * q - 1.0));
    } else if (decomp == 1) {  // barotropic: the vertical fluctuations removed (:252-274)
      for (int q = 1; q < NZ / 2; ++q) {
        c[0] = c[0] + (2.0 * c[2 * q]) * (0.5 / (2.0 * q + 1.0) - 0.5 / (2.0 * q - 1.0));
        c[2 * q - 1] = 0.0;
        c[2 * q] = 0.0;
      }
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < nc * NZ; i += blockDim.x) base[i] = tile[i];
}

__global__ void k_static_phys(Dims d, QuadDesc q, double* phys) {
  const size_t n = (size_t)d.NYA * d.NXA * d.NZA;
  for (int k = 0; k < q.st_n; ++k) {
    double* dst = phys + (size_t)q.st_var[k] * n;
    const double* src = q.st_src[k];
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
      dst[i] = q.st_prof[k] ? src[i % d.NZA] : src[i];
  }
}

struct SmagoVars {
  int n;
  int v[4];
};
// part[y][z]: the sum over x of the squares of the variables at (y, z); one CTA
// per y row, threads along z (contiguous in phys)
__global__ void k_smago_rows(Dims d, const double* phys, SmagoVars sv, double* part) {
  const int y = blockIdx.x;
  const size_t n = (size_t)d.NYA * d.NXA * d.NZA;
  for (int z = threadIdx.x; z < d.NZA; z += blockDim.x) {
    double acc = 0.0;
    for (int x = 0; x < d.NXA; ++x) {
      const size_t at = ((size_t)y * d.NXA + x) * d.NZA + z;
      double s = 0.0;
      for (int k = 0; k < sv.n; ++k) {
        const double v = phys[(size_t)sv.v[k] * n + at];
        s += v * v;
      }
      acc += s;
    }
    part[(size_t)y * d.NZA + z] = acc;
  }
}
// prof[z] = c sqrt(prof[z] + sum_y part[y][z] / NXA / NYA); the maximum to cfl_max
__global__ void k_smago_final(Dims d, const double* part, double c, double* prof, unsigned long long* cfl_max) {
  __shared__ double red[32];
  double mx = 0.0;
  for (int z = threadIdx.x; z < d.NZA; z += blockDim.x) {
    double s = 0.0;
    for (int y = 0; y < d.NYA; ++y) s += part[(size_t)y * d.NZA + z];
    const double p = c * sqrt(prof[z] + s / d.NXA / d.NYA);
    prof[z] = p;
    mx = fmax(mx, p);
  }
  if (!cfl_max) return;
  for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = mx;
  __syncthreads();
  if (threadIdx.x == 0) {
    double m2 = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) m2 = fmax(m2, red[w]);
    atomic_max_nonneg(cfl_max, m2);
  }
}

// PL_user_penalisation_mask.f90 as the reference ships it: two masks, the
// larger taken; grid labels x = (i + 2) Lx / NXAA, y = (j + 2) Ly / NYAA
// (PL_geometry.f90:138-145 with phys_iStart = 1); pi, 0.9 and 0.1 are
// single-precision literals there
__global__ void k_penal_default(Dims d, double Lx, double Ly, const double* zgrid, double* mask) {
  const size_t n = (size_t)d.NYA * d.NXA * d.NZA;
  const double pi = (double)3.14159265358979311599796346854f, c09 = (double)0.9f, c01 = (double)0.1f;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const int k = (int)(i % d.NZA);
    const size_t r = i / d.NZA;
    const int ix = (int)(r % d.NXA), iy = (int)(r / d.NXA);
    const double x = (double)(ix + 2) * Lx / d.NXA, y = (double)(iy + 2) * Ly / d.NYA, z = zgrid[k];
    const double m1 = z - (c09 + c01 * cos(5.0 * (x + y) * 2.0 * pi / Lx));
    const double cx = 6.0 + cos(2.0 * pi * x / Lx);
    const double m2 = (0.4 * exp(-(cx * cx)) / exp(-25.0)) - z;
    mask[i] = fmax(m1, m2);
  }
}
// init_penalisation (marching.f90:812-816)
__global__ void k_penal_field(size_t n, const double* mask, double strength, double width, double* out) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    double pm = tanh(width * mask[i]);
    pm = (1.0 + pm) / 2.0;
    out[i] = strength * pm;
  }
}

}  // namespace

void launch_zfilter(const Dims& d, double* Y2_var, int extract, int decomp, int y0, int ny, cudaStream_t s) {
  if (ny <= 0 || (!extract && !decomp)) return;
  const size_t sm = (size_t)kZfCols * d.NZ * sizeof(double);
  set_smem(k_zfilter, sm);
  k_zfilter<<<dim3((d.NXA + kZfCols - 1) / kZfCols, ny), 128, sm, s>>>(d, Y2_var, extract, decomp, y0);
}
void launch_static_phys(const Dims& d, const QuadDesc& q, double* phys, cudaStream_t s) {
  if (q.st_n <= 0) return;
  k_static_phys<<<4 * 148, 256, 0, s>>>(d, q, phys);
}
void launch_smago(const Dims& d, const double* phys, const int* vars, int nvars, double c, double* part, double* prof,
                  unsigned long long* cfl_max, cudaStream_t s) {
  SmagoVars sv{};
  sv.n = nvars < 4 ? nvars : 4;
  for (int k = 0; k < sv.n; ++k) sv.v[k] = vars[k];
  const int bz = d.NZA < 128 ? 128 : (d.NZA >= 512 ? 512 : (d.NZA + 31) / 32 * 32);
  k_smago_rows<<<d.NYA, bz, 0, s>>>(d, phys, sv, part);
  k_smago_final<<<1, bz, 0, s>>>(d, part, c, prof, cfl_max);
}
void launch_penal_default(const Dims& d, double Lx, double Ly, const double* zgrid, double* mask, cudaStream_t s) {
  k_penal_default<<<4 * 148, 256, 0, s>>>(d, Lx, Ly, zgrid, mask);
}
void launch_penal_field(size_t n, const double* mask, double strength, double width, double* out, cudaStream_t s) {
  k_penal_field<<<4 * 148, 256, 0, s>>>(n, mask, strength, width, out);
}
void launch_nl(const NLArgs& a, cudaStream_t s) {
  const int nsys = a.d.NXH * a.d.NYA;
  k_nl<<<(nsys + kWPB - 1) / kWPB, kWPB * 32, 0, s>>>(a);
}
void launch_solve(const SolveArgs& a, cudaStream_t s) {
  const int nsys = a.d.NXH * a.d.NYA;
  size_t sm = (size_t)kWPB * a.T * sizeof(double2);
  if (a.kl > 31 || a.kl + a.ku > 64) {
    set_smem(k_solve<true>, sm);
    k_solve<true><<<(nsys + kWPB - 1) / kWPB, kWPB * 32, sm, s>>>(a);
  } else {
    set_smem(k_solve<false>, sm);
    k_solve<false><<<(nsys + kWPB - 1) / kWPB, kWPB * 32, sm, s>>>(a);
  }
}
void launch_factor(const FactorArgs& a, cudaStream_t s) {
  if (a.nact <= 0) return;
  if (a.kl > 31) k_factor<true><<<(a.nact + kWPB - 1) / kWPB, kWPB * 32, 0, s>>>(a);
  else k_factor<false><<<(a.nact + kWPB - 1) / kWPB, kWPB * 32, 0, s>>>(a);
}
template <int RM, int RN, int G0 = 0, int G1 = 0, int G2 = 0>
static void launch_rhs_tiles(const SolveArgs& a, const NLArgs& n, cudaStream_t s) {
  const int nsys = a.d.NXH * a.d.NYA;
  const size_t sm = (size_t)kRhsSys * a.rhs_win_max * sizeof(double2);
  set_smem(k_rhs_tiles<RM, RN, G0, G1, G2>, sm);
  const dim3 g((nsys + kRhsSys - 1) / kRhsSys, (a.T + kTileRows - 1) / kTileRows);
  k_rhs_tiles<RM, RN, G0, G1, G2><<<g, kTileRows, sm, s>>>(a, n);
}
// slot widths of the groups of a grouped operator (0 past its last group)
static void group_widths(const DevGEll& G, int w[3]) {
  w[0] = w[1] = w[2] = 0;
  for (int k = 0; k < G.width; ++k)
    if (G.slot_grp[k] < 3) ++w[G.slot_grp[k]];
}
// threads of a one-CTA-per-system kernel: one per row up to kRhsThreads (a
// system of 64 rows takes 2 warps, not 8 of which 6 would idle)
static int rows_threads(int T) { return std::min(kRhsThreads, std::max(32, (T + 31) / 32 * 32)); }
void launch_rhs_nl(const SolveArgs& a, const NLArgs& n, cudaStream_t s) {
  if (a.work2 && a.rhs_win && a.row_pos) {
    if (!a.generic_tiles && a.NLg.valid && a.NLg.ngroups == 3 && a.Mw.width <= 4) {
      int w[3];
      group_widths(a.NLg, w);
      // the plane-layer recipes' NL operator: groups i kx, i ky, 1 of widths 3, 3, 2;
      // with a penalisation drag (- Iz.Iz.Gu beside - Iz.uw) 3, 3, 5; with a
      // second flux in each derivative group (an eddy-viscosity term) 6, 6, 2
      if (w[0] == 3 && w[1] == 3 && w[2] == 2) return launch_rhs_tiles<4, 8, 3, 3, 2>(a, n, s);
      if (w[0] == 3 && w[1] == 3 && w[2] == 5) return launch_rhs_tiles<4, 11, 3, 3, 5>(a, n, s);
      if (w[0] == 6 && w[1] == 6 && w[2] == 2) return launch_rhs_tiles<4, 14, 6, 6, 2>(a, n, s);
    }
    if (a.Mw.width <= 4 && a.NLw.width <= 8) return launch_rhs_tiles<4, 8>(a, n, s);
    if (a.Mw.width <= 8 && a.NLw.width <= 16) return launch_rhs_tiles<8, 16>(a, n, s);
  }
  const int nsys = a.d.NXH * a.d.NYA;
  const size_t sm = ((size_t)n.nq * a.d.NZ + a.T) * sizeof(double2);
  set_smem(k_rhs_nl, sm);
  k_rhs_nl<<<nsys, rows_threads(a.T), sm, s>>>(a, n);
}
void launch_subst(const SolveArgs& a, cudaStream_t s) {
  if (a.nact <= 0) return;
  if (a.work2) {
    if (a.nblk > 0) {
      const int kv = a.kl + a.ku, grid = (a.nblk + kTpbThreads - 1) / kTpbThreads;
      // band (kl, kl+ku) = (9, 23) of the plane-layer recipes compiled, any other
      // band within (15, 31) through the run-time-band kernel
      if (!a.subst_rt && a.kl == 9 && kv == 23 && a.ldab == 34) {
        const size_t sm = (size_t)kTpbThreads * 24 * sizeof(double2);
        set_smem(k_subst_tpb<9, 23, 34>, sm);
        k_subst_tpb<9, 23, 34><<<grid, kTpbThreads, sm, s>>>(a);
      } else {
        const size_t sm = (size_t)kTpbThreads * 32 * sizeof(double2);
        set_smem(k_subst_tpb_rt<15, 31>, sm);
        k_subst_tpb_rt<15, 31><<<grid, kTpbThreads, sm, s>>>(a);
      }
    }
    return;
  }
  // whole systems (no class split): one warp per system
  const size_t sm = (size_t)kWPBr * kNBUF * kCW * a.ring_cols * sizeof(double);
  set_smem(k_subst_real<32>, sm);
  k_subst_real<32><<<(a.nact + kWPBr - 1) / kWPBr, kWPBr * 32, sm, s>>>(a);
}
bool subst_multi_supported(const SolveArgs& a) {
  return a.work2 && a.nblk > 0 && a.kl == 9 && a.kl + a.ku == 23 && a.ldab == 34;
}
void launch_subst_multi(const SolveArgs* d_args, const long long* d_prefix, int nmem, long long total,
                        cudaStream_t s) {
  if (total <= 0) return;
  const size_t sm = (size_t)kTpbThreads * 24 * sizeof(double2);
  set_smem(k_subst_tpb_multi<9, 23, 34>, sm);
  static int nct = 0;
  if (!nct) nct = persistent_ctas(k_subst_tpb_multi<9, 23, 34>, kTpbThreads, sm);
  const long long need = (total + kTpbThreads - 1) / kTpbThreads;
  k_subst_tpb_multi<9, 23, 34><<<(int)std::min<long long>(nct, need), kTpbThreads, sm, s>>>(d_args, d_prefix, nmem,
                                                                                          total);
}
void launch_kstd_out(const SolveArgs& a, cudaStream_t s) {
  if (a.nact <= 0) return;
  if (a.work2 && !a.Kstd_out) return;  // solution already in out, no K_std in the last stage
  if (a.work2 && a.tile_win && a.Lw.valid && a.Lw.width <= kLW) {
    const size_t sm = (size_t)kTileSys * a.tile_lwin_max * sizeof(double2);
    const dim3 g((a.T + kTileRows - 1) / kTileRows, (a.nact + kTileSys - 1) / kTileSys);
    int w[4] = {0, 0, 0, 0};
    for (int k = 0; k < a.Lw.width; ++k)
      if (a.Lw.slot_grp[k] < 4) ++w[a.Lw.slot_grp[k]];
    if (!a.generic_tiles && a.Lw.ngroups == 4 && w[0] == 4 && w[1] == 6 && w[2] == 3 && w[3] == 3) {
      // the plane-layer recipes' L: (kx^2 + ky^2), 1, kx, ky groups
      set_smem(k_kstd_tiles<4, 6, 3, 3>, sm);
      k_kstd_tiles<4, 6, 3, 3><<<g, kTileRows, sm, s>>>(a);
      return;
    }
    set_smem(k_kstd_tiles<>, sm);
    k_kstd_tiles<><<<g, kTileRows, sm, s>>>(a);
    return;
  }
  const size_t smx = (size_t)a.T * sizeof(double2);
  if (smx > 48 * 1024) set_smem(k_kstd_out, smx);
  k_kstd_out<<<a.nact, rows_threads(a.T), smx, s>>>(a);
}
void launch_solve_real(const SolveArgs& a, const NLArgs& n, cudaStream_t s) {
  launch_rhs_nl(a, n, s);
  launch_subst(a, s);
  launch_kstd_out(a, s);
}
void launch_factor_real(const FactorArgs& a, cudaStream_t s) {
  if (a.nact <= 0) return;
  if (a.tpb) {
    const int nb = a.ncls * a.nact;
    // the shared-memory window kernel when a warp's (or at least one thread's)
    // windows fit in a CTA's shared memory, else the in-place kernel
    int dev = 0, smax = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&smax, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    const size_t wbytes = (size_t)(a.kl + a.ku + 2) * a.ldab * sizeof(double);
    const int nt = (int)std::min<size_t>(32, (size_t)smax / wbytes);
    if (a.window && a.kl <= kFacKl && nt >= 1) {
      if (a.M.ngroups <= 8 && a.L.ngroups <= 8)
        k_assemble_tpb<8><<<(nb + kTpbThreads - 1) / kTpbThreads, kTpbThreads, 0, s>>>(a);
      else
        k_assemble_tpb<kMaxGroups><<<(nb + kTpbThreads - 1) / kTpbThreads, kTpbThreads, 0, s>>>(a);
      set_smem(k_factor_win, (size_t)nt * wbytes);
      k_factor_win<<<(nb + nt - 1) / nt, nt, (size_t)nt * wbytes, s>>>(a);
    } else {
      k_factor_tpb<<<(nb + kTpbThreads - 1) / kTpbThreads, kTpbThreads, 0, s>>>(a);
    }
    if (a.cmask && a.ldab <= 64 && a.kl + a.ku <= 32 && a.kl <= 32) {
      cudaMemsetAsync(a.cmask, 0, (size_t)a.Tc * sizeof(unsigned long long), s);
      k_mask_cols<<<dim3((nb + 31) / 32, (a.Tc + 7) / 8), 256, 0, s>>>(a);
      k_mask_rows<<<(a.Tc + 127) / 128, 128, 0, s>>>(a);
    }
    return;
  }
  k_factor_real<<<dim3((a.nact + kWPB - 1) / kWPB, a.ncls), kWPB * 32, 0, s>>>(a);
}
void launch_zero_step(const ZeroArgs& a, cudaStream_t s) {
  if (a.nsys <= 0) return;
  size_t sm = 8;
  for (int i = 0; i < a.nsys; ++i) sm = std::max(sm, (size_t)a.sys[i].T * (1 + a.sys[i].ldab) * sizeof(double));
  set_smem(k_zero_step, sm);
  k_zero_step<<<a.nsys, 32, sm, s>>>(a);
}
void launch_zero_factor(const ZeroArgs& a, cudaStream_t s) {
  if (a.nsys <= 0) return;
  k_zero_factor<<<a.nsys, 32, 0, s>>>(a);
}
void launch_full_dz(const Dims& d, const double2* state, int T, const int* tab_t, const double* tab_v, double dsca,
                    int order, double gap, double2* out, cudaStream_t s) {
  k_full_dz<<<grid1d((size_t)d.NXH * d.NYA, 128), 128, 0, s>>>(d, state, T, tab_t, tab_v, dsca, order, gap, out);
}
void launch_zero_dz(int NZ, const double* state, const int* tab_t, const double* tab_v, double dsca, int order,
                    double gap, double* out, cudaStream_t s) {
  k_zero_dz<<<1, 32, 0, s>>>(NZ, state, tab_t, tab_v, dsca, order, gap, out);
}
void launch_usr_slice(const Dims& d, const double* phys, int kind, int k, const double* wz, double* out,
                      cudaStream_t s) {
  k_usr_slice<<<1024, 256, 0, s>>>(d, phys, kind, k, wz, out);
}
void launch_usr_profile(const Dims& d, const double* phys, double* out, cudaStream_t s) {
  k_usr_profile<<<d.NZA, 256, 0, s>>>(d, phys, out);
}
void launch_phys_product(size_t n, const double* a, const double* b, double* out, cudaStream_t s) {
  k_phys_product<<<1024, 256, 0, s>>>(n, a, b, out);
}
void launch_transpose_xy(const Dims& d, const double* in, double* out, int to_file, cudaStream_t s) {
  k_transpose_xy<<<1024, 256, 0, s>>>(d, in, out, to_file);
}
void launch_galerkin_insert(const Dims& d, const double2* spec, int T, const int* var_pos, int nc, const double* sq,
                            const int* sq_col, double2* field, cudaStream_t s) {
  k_galerkin_insert<<<grid1d((size_t)d.NXH * d.NYA, 128), 128, 0, s>>>(d, spec, T, var_pos, nc, sq, sq_col, field);
}
void launch_cheb_extract(const Dims& d, const double2* field, int T, const int* tab_t, const double* tab_v,
                         double2* spec, cudaStream_t s) {
  k_cheb_extract<<<grid1d((size_t)d.NXH * d.NYA * d.NZ, 256), 256, 0, s>>>(d, field, T, tab_t, tab_v, spec);
}
void launch_check_finite(const double2* x, size_t n, unsigned int* flags, cudaStream_t s) {
  k_check_finite<<<1024, 256, 0, s>>>(x, n, flags);
}

}  // namespace coral
