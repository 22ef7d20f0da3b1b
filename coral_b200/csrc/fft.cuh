// Shared-memory FFTs for the transform kernels (sm_100a, FP64).
//
// A CTA transforms a batch of lines held contiguously in shared memory
// (line-major, line stride N) with a self-sorting Stockham scheme of radix 4, 3
// and 2 stages (all grid sizes of the plane-layer problems are 2^a 3^b).  The
// twiddles exp(-2 pi i k / N) come from a table computed on the host in long
// double.  Real transforms pack two real lines into one complex line.
#pragma once
#include <cuda_runtime.h>

namespace coral {

struct FftPlan {
  int N;
  int nst;
  int radix[16];
  const double2* tw;  // tw[k] = exp(-2 pi i k / N), k < N
};

__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }
__device__ __forceinline__ double2 cscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
// multiply by -i (forward) or +i (inverse)
template <bool INV>
__device__ __forceinline__ double2 mul_mi(double2 a) {
  return INV ? make_double2(-a.y, a.x) : make_double2(a.y, -a.x);
}

// sin(pi/3), from the mathematics
#define CORAL_SIN60 0.86602540378443864676372317075293618

// Ping-pong batched FFT of nl lines of length p.N stored in A (line stride LS)
// with a plan chosen at run time (lengths without a compile-time plan).  B is
// scratch of the same size.  Returns the buffer that holds the result.
// INV = false: exp(-i), INV = true: exp(+i); no normalisation.
// Must be called by all threads of the CTA (contains __syncthreads).
template <bool INV>
__device__ double2* fft_lines(double2* A, double2* B, int nl, int LS, const FftPlan& p) {
  double2* src = A;
  double2* dst = B;
  const int N = p.N;
  int Ns = 1;
  for (int s = 0; s < p.nst; ++s) {
    const int R = p.radix[s];
    const int nb = N / R;
    const int tstride = N / (Ns * R);
    const int total = nl * nb;
    for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
      const int line = idx / nb;
      const int j = idx - line * nb;
      const int k = j % Ns;
      const double2* sl = src + line * LS;
      double2* dl = dst + line * LS;
      const int od = (j / Ns) * Ns * R + k;
      if (R == 4) {
        double2 a0 = sl[j], a1 = sl[j + nb], a2 = sl[j + 2 * nb], a3 = sl[j + 3 * nb];
        if (Ns > 1) {
          double2 w1 = p.tw[k * tstride], w2 = p.tw[2 * k * tstride], w3 = p.tw[3 * k * tstride];
          if (INV) { w1 = cconj(w1); w2 = cconj(w2); w3 = cconj(w3); }
          a1 = cmul(a1, w1); a2 = cmul(a2, w2); a3 = cmul(a3, w3);
        }
        double2 t0 = cadd(a0, a2), t1 = csub(a0, a2), t2 = cadd(a1, a3), t3 = mul_mi<INV>(csub(a1, a3));
        dl[od] = cadd(t0, t2);
        dl[od + Ns] = cadd(t1, t3);
        dl[od + 2 * Ns] = csub(t0, t2);
        dl[od + 3 * Ns] = csub(t1, t3);
      } else if (R == 3) {
        double2 a0 = sl[j], a1 = sl[j + nb], a2 = sl[j + 2 * nb];
        if (Ns > 1) {
          double2 w1 = p.tw[k * tstride], w2 = p.tw[2 * k * tstride];
          if (INV) { w1 = cconj(w1); w2 = cconj(w2); }
          a1 = cmul(a1, w1); a2 = cmul(a2, w2);
        }
        double2 t = cadd(a1, a2), d = csub(a1, a2);
        double2 m = make_double2(a0.x - 0.5 * t.x, a0.y - 0.5 * t.y);
        // forward: y1 = m - i s d, y2 = m + i s d ; inverse: s -> -s
        const double sd = INV ? -CORAL_SIN60 : CORAL_SIN60;
        double2 isd = make_double2(-sd * d.y, sd * d.x);  // i*s*d
        dl[od] = cadd(a0, t);
        dl[od + Ns] = csub(m, isd);
        dl[od + 2 * Ns] = cadd(m, isd);
      } else {  // R == 2
        double2 a0 = sl[j], a1 = sl[j + nb];
        if (Ns > 1) {
          double2 w1 = p.tw[k * tstride];
          if (INV) w1 = cconj(w1);
          a1 = cmul(a1, w1);
        }
        dl[od] = cadd(a0, a1);
        dl[od + Ns] = csub(a0, a1);
      }
    }
    __syncthreads();
    double2* t = src;
    src = dst;
    dst = t;
    Ns *= R;
  }
  return src;
}

// ---- compile-time plans: register passes ----------------------------------------
// With the length N known at compile time the transform runs as a few passes of
// radix 24, 18, 16, 9, 8, 4, 3 or 2 (in the three-pass plans odd radices come
// first: their strided stores in the first pass hit distinct shared-memory banks;
// the two-pass plans trade that for one pass fewer).  Each thread computes whole
// radix-R butterflies in registers: it loads its R inputs, applies the twiddles,
// waits for every thread to have loaded (so the pass can write in place), and
// stores its R outputs at their Stockham (self-sorting) positions.  Only one
// line buffer is needed.
struct PlanR {
  int nst;
  int r[12];
};
__host__ __device__ constexpr PlanR make_planr(int N) {
  PlanR p{0, {}};
  int n = N, a = 0, b = 0;
  while (n % 3 == 0) { n /= 3; ++b; }
  while (n % 2 == 0) { n /= 2; ++a; }
  if (n != 1) return PlanR{0, {}};
  for (; b >= 2; b -= 2) p.r[p.nst++] = 9;
  if (b == 1) p.r[p.nst++] = 3;
  while (a > 0) {
    if (a == 6) { p.r[p.nst++] = 8; p.r[p.nst++] = 8; a = 0; }
    else if (a == 5) { p.r[p.nst++] = 8; p.r[p.nst++] = 4; a = 0; }
    else if (a >= 4) { p.r[p.nst++] = 16; a -= 4; }
    else if (a == 3) { p.r[p.nst++] = 8; a = 0; }
    else if (a == 2) { p.r[p.nst++] = 4; a = 0; }
    else { p.r[p.nst++] = 2; a = 0; }
  }
  return p;
}

// Two-pass plans (more registers per thread, one barrier pair fewer):
// 288 = 18 x 16, 576 = 24 x 24; other lengths keep make_planr.
__host__ __device__ constexpr PlanR make_planr2(int N) {
  if (N == 288) return PlanR{2, {18, 16}};
  if (N == 576) return PlanR{2, {24, 24}};
  return make_planr(N);
}
// plan variant PV: 0 = make_planr, 1 = make_planr2
__host__ __device__ constexpr PlanR plan_of(int N, int PV) { return PV ? make_planr2(N) : make_planr(N); }

// cos / sin of 2 pi m / 16 and 2 pi m / 9, from the mathematics (40-digit values)
#define CORAL_C16_1 0.923879532511286756128183189396788287   // cos(pi/8)
#define CORAL_S16_1 0.382683432365089771728459984030398867   // sin(pi/8)
#define CORAL_SQRT1_2 0.707106781186547524400844362104849039 // cos(pi/4)
#define CORAL_C9_1 0.766044443118978035202392650555416674    // cos(2 pi/9)
#define CORAL_S9_1 0.642787609686539326322643409907263433    // sin(2 pi/9)
#define CORAL_C9_2 0.173648177666930348851716626769314796    // cos(4 pi/9)
#define CORAL_S9_2 0.984807753012208059366743024589523014    // sin(4 pi/9)
#define CORAL_C9_4 (-0.93969262078590838405410927732473147)  // cos(8 pi/9)
#define CORAL_S9_4 0.342020143325668733044099614682259581    // sin(8 pi/9)

// cos / sin of 2 pi m / 18 and 2 pi m / 24 (m = 0, 1, ...), from the mathematics
__device__ constexpr double kC18[9] = {1.0, 0.93969262078590838405410927732473147, 0.766044443118978035202392650555416674,
                                       0.5, 0.173648177666930348851716626769314796, -0.173648177666930348851716626769314796,
                                       -0.5, -0.766044443118978035202392650555416674, -0.93969262078590838405410927732473147};
__device__ constexpr double kS18[9] = {0.0, 0.342020143325668733044099614682259581, 0.642787609686539326322643409907263433,
                                       0.866025403784438646763723170752936183, 0.984807753012208059366743024589523014,
                                       0.984807753012208059366743024589523014, 0.866025403784438646763723170752936183,
                                       0.642787609686539326322643409907263433, 0.342020143325668733044099614682259581};
__device__ constexpr double kC24[15] = {1.0, 0.965925826289068286749743199728897368, 0.866025403784438646763723170752936183,
                                        0.707106781186547524400844362104849039, 0.5, 0.258819045102520762348898837624048328,
                                        0.0, -0.258819045102520762348898837624048328, -0.5,
                                        -0.707106781186547524400844362104849039, -0.866025403784438646763723170752936183,
                                        -0.965925826289068286749743199728897368, -1.0,
                                        -0.965925826289068286749743199728897368, -0.866025403784438646763723170752936183};
__device__ constexpr double kS24[15] = {0.0, 0.258819045102520762348898837624048328, 0.5,
                                        0.707106781186547524400844362104849039, 0.866025403784438646763723170752936183,
                                        0.965925826289068286749743199728897368, 1.0, 0.965925826289068286749743199728897368,
                                        0.866025403784438646763723170752936183, 0.707106781186547524400844362104849039, 0.5,
                                        0.258819045102520762348898837624048328, 0.0, -0.258819045102520762348898837624048328,
                                        -0.5};

// a * exp(-i t) (forward) or a * exp(+i t) (inverse), given c = cos t, s = sin t
template <bool INV>
__device__ __forceinline__ double2 rot(double2 a, double c, double s) {
  return INV ? make_double2(a.x * c - a.y * s, a.x * s + a.y * c) : make_double2(a.x * c + a.y * s, a.y * c - a.x * s);
}

template <bool INV>
__device__ __forceinline__ void dft3(double2& a0, double2& a1, double2& a2) {
  const double2 t = cadd(a1, a2), d = csub(a1, a2);
  const double2 m = make_double2(a0.x - 0.5 * t.x, a0.y - 0.5 * t.y);
  const double sd = INV ? -CORAL_SIN60 : CORAL_SIN60;
  const double2 isd = make_double2(-sd * d.y, sd * d.x);  // i s d
  a0 = cadd(a0, t);
  a1 = csub(m, isd);
  a2 = cadd(m, isd);
}
template <bool INV>
__device__ __forceinline__ void dft4(double2& a0, double2& a1, double2& a2, double2& a3) {
  const double2 t0 = cadd(a0, a2), t1 = csub(a0, a2), t2 = cadd(a1, a3), t3 = mul_mi<INV>(csub(a1, a3));
  a0 = cadd(t0, t2);
  a1 = cadd(t1, t3);
  a2 = csub(t0, t2);
  a3 = csub(t1, t3);
}

// in-register DFT of length R, natural order in and out
template <int R, bool INV>
__device__ __forceinline__ void dft(double2 (&x)[R]) {
  if constexpr (R == 2) {
    const double2 t = x[0];
    x[0] = cadd(t, x[1]);
    x[1] = csub(t, x[1]);
  } else if constexpr (R == 3) {
    dft3<INV>(x[0], x[1], x[2]);
  } else if constexpr (R == 4) {
    dft4<INV>(x[0], x[1], x[2], x[3]);
  } else if constexpr (R == 8) {
    // n = 2 n1 + n2, k = k1 + 4 k2
    dft4<INV>(x[0], x[2], x[4], x[6]);
    dft4<INV>(x[1], x[3], x[5], x[7]);
    x[3] = rot<INV>(x[3], CORAL_SQRT1_2, CORAL_SQRT1_2);
    x[5] = mul_mi<INV>(x[5]);
    x[7] = rot<INV>(x[7], -CORAL_SQRT1_2, CORAL_SQRT1_2);
    double2 y[8];
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1) {
      y[k1] = cadd(x[2 * k1], x[2 * k1 + 1]);
      y[k1 + 4] = csub(x[2 * k1], x[2 * k1 + 1]);
    }
#pragma unroll
    for (int k = 0; k < 8; ++k) x[k] = y[k];
  } else if constexpr (R == 9) {
    // n = 3 n1 + n2, k = k1 + 3 k2
    dft3<INV>(x[0], x[3], x[6]);
    dft3<INV>(x[1], x[4], x[7]);
    dft3<INV>(x[2], x[5], x[8]);
    // A_{n2}[k1] sits in x[n2 + 3 k1]; twiddle by w9^(n2 k1)
    x[4] = rot<INV>(x[4], CORAL_C9_1, CORAL_S9_1);
    x[7] = rot<INV>(x[7], CORAL_C9_2, CORAL_S9_2);
    x[5] = rot<INV>(x[5], CORAL_C9_2, CORAL_S9_2);
    x[8] = rot<INV>(x[8], CORAL_C9_4, CORAL_S9_4);
    dft3<INV>(x[0], x[1], x[2]);  // k1 = 0 -> X[0], X[3], X[6]
    dft3<INV>(x[3], x[4], x[5]);  // k1 = 1 -> X[1], X[4], X[7]
    dft3<INV>(x[6], x[7], x[8]);  // k1 = 2 -> X[2], X[5], X[8]
    double2 y[9];
#pragma unroll
    for (int k1 = 0; k1 < 3; ++k1)
#pragma unroll
      for (int k2 = 0; k2 < 3; ++k2) y[k1 + 3 * k2] = x[3 * k1 + k2];
#pragma unroll
    for (int k = 0; k < 9; ++k) x[k] = y[k];
  } else if constexpr (R == 18) {
    // n = 2 n1 + n2, k = k1 + 9 k2: two 9-point DFTs, twiddles w18^k1, butterflies
    double2 e[9], o[9];
#pragma unroll
    for (int n1 = 0; n1 < 9; ++n1) {
      e[n1] = x[2 * n1];
      o[n1] = x[2 * n1 + 1];
    }
    dft<9, INV>(e);
    dft<9, INV>(o);
#pragma unroll
    for (int k1 = 1; k1 < 9; ++k1) o[k1] = rot<INV>(o[k1], kC18[k1], kS18[k1]);
#pragma unroll
    for (int k1 = 0; k1 < 9; ++k1) {
      x[k1] = cadd(e[k1], o[k1]);
      x[k1 + 9] = csub(e[k1], o[k1]);
    }
  } else if constexpr (R == 24) {
    // n = 3 n1 + n2, k = k1 + 8 k2: three 8-point DFTs, twiddles w24^(n2 k1), 3-point DFTs
    double2 a0[8], a1[8], a2[8];
#pragma unroll
    for (int n1 = 0; n1 < 8; ++n1) {
      a0[n1] = x[3 * n1];
      a1[n1] = x[3 * n1 + 1];
      a2[n1] = x[3 * n1 + 2];
    }
    dft<8, INV>(a0);
    dft<8, INV>(a1);
    dft<8, INV>(a2);
#pragma unroll
    for (int k1 = 1; k1 < 8; ++k1) {
      a1[k1] = rot<INV>(a1[k1], kC24[k1], kS24[k1]);
      a2[k1] = rot<INV>(a2[k1], kC24[2 * k1], kS24[2 * k1]);
    }
#pragma unroll
    for (int k1 = 0; k1 < 8; ++k1) {
      dft3<INV>(a0[k1], a1[k1], a2[k1]);
      x[k1] = a0[k1];
      x[k1 + 8] = a1[k1];
      x[k1 + 16] = a2[k1];
    }
  } else if constexpr (R == 16) {
    // n = 4 n1 + n2, k = k1 + 4 k2
#pragma unroll
    for (int n2 = 0; n2 < 4; ++n2) dft4<INV>(x[n2], x[n2 + 4], x[n2 + 8], x[n2 + 12]);
    // A_{n2}[k1] sits in x[n2 + 4 k1]; twiddle by w16^(n2 k1)
    x[5] = rot<INV>(x[5], CORAL_C16_1, CORAL_S16_1);      // 1
    x[9] = rot<INV>(x[9], CORAL_SQRT1_2, CORAL_SQRT1_2);  // 2
    x[13] = rot<INV>(x[13], CORAL_S16_1, CORAL_C16_1);    // 3
    x[6] = rot<INV>(x[6], CORAL_SQRT1_2, CORAL_SQRT1_2);  // 2
    x[10] = mul_mi<INV>(x[10]);                            // 4
    x[14] = rot<INV>(x[14], -CORAL_SQRT1_2, CORAL_SQRT1_2);  // 6
    x[7] = rot<INV>(x[7], CORAL_S16_1, CORAL_C16_1);      // 3
    x[11] = rot<INV>(x[11], -CORAL_SQRT1_2, CORAL_SQRT1_2);  // 6
    x[15] = rot<INV>(x[15], -CORAL_C16_1, -CORAL_S16_1);  // 9
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1) dft4<INV>(x[4 * k1], x[4 * k1 + 1], x[4 * k1 + 2], x[4 * k1 + 3]);
    double2 y[16];
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1)
#pragma unroll
      for (int k2 = 0; k2 < 4; ++k2) y[k1 + 4 * k2] = x[4 * k1 + k2];
#pragma unroll
    for (int k = 0; k < 16; ++k) x[k] = y[k];
  }
}

// Twiddles of the second pass of a two-pass plan N = R0 x R1, laid out [k][r - 1]
// (k < R0, 1 <= r < R1): t[k (R1 - 1) + r - 1] = exp(-2 pi i r k / N).  For a
// fixed r, consecutive k are R1 - 1 16-byte words apart, an odd number for the
// even R1 of the two-pass plans, so the 16-byte reads of 8 consecutive k fall in
// 8 distinct bank groups (the N-entry table read at r k conflicts up to 8-way).
template <int N, int PV>
__host__ __device__ constexpr int tw_pass2_len() {
  return plan_of(N, PV).nst == 2 ? plan_of(N, PV).r[0] * (plan_of(N, PV).r[1] - 1) : 0;
}
template <int N, int PV>
__device__ __forceinline__ void build_tw_pass2(double2* t, const double2* tw) {
  constexpr PlanR P = plan_of(N, PV);
  static_assert(P.nst == 2 && (P.r[1] % 2) == 0, "two-pass plan with an even second radix");
  constexpr int R0 = P.r[0], R1 = P.r[1];
  for (int i = threadIdx.x; i < R0 * (R1 - 1); i += blockDim.x) {
    const int k = i / (R1 - 1), r = i - k * (R1 - 1) + 1;
    t[i] = tw[r * k];  // N = R0 R1: the pass's twiddle stride is 1
  }
}

// One in-place pass of radix R over nl lines (line stride LS) by NT threads;
// NLMAX bounds nl (registers hold ceil(NLMAX N / (R NT)) butterflies per thread).
// TWL: tw is the [k][r - 1] table of build_tw_pass2 (second pass of a two-pass plan).
template <int N, int R, int Ns, bool INV, int NT, int NLMAX, bool TWL = false>
__device__ __forceinline__ void fft_pass(double2* A, int nl, int LS, const double2* __restrict__ tw) {
  constexpr int NB = N / R;               // butterflies per line
  constexpr int TS = N / (Ns * R);        // twiddle stride
  constexpr int BPT = (NLMAX * NB + NT - 1) / NT;
  const int total = nl * NB;
  double2 v[BPT][R];
#pragma unroll
  for (int i = 0; i < BPT; ++i) {
    const int b = threadIdx.x + i * NT;
    if (b < total) {
      const int line = b / NB, j = b - line * NB;
      const double2* sl = A + line * LS + j;
#pragma unroll
      for (int r = 0; r < R; ++r) v[i][r] = sl[r * NB];
      if constexpr (Ns > 1) {
        const int k = j % Ns;
#pragma unroll
        for (int r = 1; r < R; ++r) {
          double2 w = TWL ? tw[k * (R - 1) + r - 1] : tw[r * k * TS];
          if (INV) w = cconj(w);
          v[i][r] = cmul(v[i][r], w);
        }
      }
      dft<R, INV>(v[i]);
    }
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < BPT; ++i) {
    const int b = threadIdx.x + i * NT;
    if (b < total) {
      const int line = b / NB, j = b - line * NB;
      double2* dl = A + line * LS + (j / Ns) * Ns * R + (j % Ns);
#pragma unroll
      for (int r = 0; r < R; ++r) dl[r * Ns] = v[i][r];
    }
  }
  __syncthreads();
}

// The first pass (Ns = 1, no twiddles) with its inputs produced by ld(line, k)
// (k = position in the line) instead of read from shared memory; it writes its
// outputs in place into A, which nothing reads during the pass, so it needs no
// barrier between loads and stores.
// LINE_FAST: consecutive threads take consecutive lines at the same position
// (so that interleaved lines of a global array load together); otherwise
// consecutive positions of one line.
template <int N, int R, bool INV, int NT, int NLMAX, bool LINE_FAST, class Load>
__device__ __forceinline__ void fft_pass_first(double2* A, int nl, int LS, Load&& ld) {
  constexpr int NB = N / R;
  constexpr int BPT = (NLMAX * NB + NT - 1) / NT;
  const int total = nl * NB;
#pragma unroll
  for (int i = 0; i < BPT; ++i) {
    const int b = threadIdx.x + i * NT;
    if (b < total) {
      const int line = LINE_FAST ? b % nl : b / NB;
      const int j = LINE_FAST ? b / nl : b - line * NB;
      double2 v[R];
#pragma unroll
      for (int r = 0; r < R; ++r) v[r] = ld(line, j + r * NB);
      dft<R, INV>(v);
      double2* dl = A + line * LS + j * R;
#pragma unroll
      for (int r = 0; r < R; ++r) dl[r] = v[r];
    }
  }
  __syncthreads();
}

template <int N, int S, int Ns, bool INV, int NT, int NLMAX, int PV = 0, bool TWL = false>
__device__ __forceinline__ void fft_passes(double2* A, int nl, int LS, const double2* tw) {
  constexpr PlanR P = plan_of(N, PV);
  static_assert(!TWL || P.nst == 2, "the pass-2 twiddle table belongs to two-pass plans");
  if constexpr (S < P.nst) {
    constexpr int R = P.r[S];
    fft_pass<N, R, Ns, INV, NT, NLMAX, TWL>(A, nl, LS, tw);
    fft_passes<N, S + 1, Ns * R, INV, NT, NLMAX, PV, TWL>(A, nl, LS, tw);
  }
}

// Batched FFT of nl <= NLMAX lines (line stride LS) by NT threads: compile-time
// length NC in place in A (B unused), or the runtime plan (NC == 0) ping-ponging
// through B.  Returns the buffer holding the result.  The caller synchronises
// before (inputs written) and may read the result directly after.
// The same with the inputs produced by ld(line, k) (see fft_pass_first); the
// caller need not synchronise before.  Runtime plans stage the inputs in A first.
// TWL: p.tw is the table of build_tw_pass2 (compiled two-pass plans only).
template <int NC, bool INV, int NT, int NLMAX, bool LINE_FAST = false, int PV = 0, bool TWL = false, class Load>
__device__ __forceinline__ double2* fft_lines_ld(double2* A, double2* B, int nl, int LS, const FftPlan& p,
                                                 Load&& ld) {
  if constexpr (NC == 0) {
    for (int idx = threadIdx.x; idx < nl * p.N; idx += blockDim.x) {
      const int line = idx / p.N, k = idx - line * p.N;
      A[line * LS + k] = ld(line, k);
    }
    __syncthreads();
    return fft_lines<INV>(A, B, nl, LS, p);
  } else {
    constexpr PlanR P = plan_of(NC, PV);
    static_assert(P.nst > 0, "transform length must be 2^a 3^b");
    fft_pass_first<NC, P.r[0], INV, NT, NLMAX, LINE_FAST>(A, nl, LS, ld);
    fft_passes<NC, 1, P.r[0], INV, NT, NLMAX, PV, TWL>(A, nl, LS, p.tw);
    return A;
  }
}

template <int NC, bool INV, int NT, int NLMAX>
__device__ __forceinline__ double2* fft_lines_n(double2* A, double2* B, int nl, int LS, const FftPlan& p) {
  if constexpr (NC == 0) {
    return fft_lines<INV>(A, B, nl, LS, p);
  } else {
    static_assert(make_planr(NC).nst > 0, "transform length must be 2^a 3^b");
    fft_passes<NC, 0, 1, INV, NT, NLMAX>(A, nl, LS, p.tw);
    return A;
  }
}

}  // namespace coral
