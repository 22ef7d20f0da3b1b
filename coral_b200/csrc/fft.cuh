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

// In-place-by-pingpong batched FFT of nl lines of length p.N stored in A (line
// stride p.N).  B is scratch of the same size.  Returns the buffer that holds
// the result.  INV = false: exp(-i), INV = true: exp(+i); no normalisation.
// Must be called by all threads of the CTA (contains __syncthreads).
template <bool INV>
__device__ double2* fft_lines(double2* A, double2* B, int nl, const FftPlan& p) {
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
      const double2* sl = src + line * N;
      double2* dl = dst + line * N;
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

// ---- compile-time plans --------------------------------------------------------
// The same Stockham scheme with the transform length known at compile time:
// radices, strides and all index arithmetic fold into constants.
struct PlanC {
  int nst;
  int r[16];
};
__host__ __device__ constexpr PlanC make_planc(int N) {
  PlanC p{0, {}};
  int n = N;
  while (n % 4 == 0) { p.r[p.nst++] = 4; n /= 4; }
  while (n % 3 == 0) { p.r[p.nst++] = 3; n /= 3; }
  while (n % 2 == 0) { p.r[p.nst++] = 2; n /= 2; }
  return p;
}

template <int N, int R, int Ns, bool INV>
__device__ __forceinline__ void fft_stage_t(const double2* __restrict__ src, double2* __restrict__ dst, int nl,
                                            const double2* __restrict__ tw) {
  constexpr int nb = N / R;
  constexpr int tstride = N / (Ns * R);
  const int total = nl * nb;
  for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
    const int line = idx / nb;
    const int j = idx - line * nb;
    const int k = j % Ns;
    const double2* sl = src + line * N;
    double2* dl = dst + line * N;
    const int od = (j / Ns) * Ns * R + k;
    if constexpr (R == 4) {
      double2 a0 = sl[j], a1 = sl[j + nb], a2 = sl[j + 2 * nb], a3 = sl[j + 3 * nb];
      if constexpr (Ns > 1) {
        double2 w1 = tw[k * tstride], w2 = tw[2 * k * tstride], w3 = tw[3 * k * tstride];
        if (INV) { w1 = cconj(w1); w2 = cconj(w2); w3 = cconj(w3); }
        a1 = cmul(a1, w1); a2 = cmul(a2, w2); a3 = cmul(a3, w3);
      }
      double2 t0 = cadd(a0, a2), t1 = csub(a0, a2), t2 = cadd(a1, a3), t3 = mul_mi<INV>(csub(a1, a3));
      dl[od] = cadd(t0, t2);
      dl[od + Ns] = cadd(t1, t3);
      dl[od + 2 * Ns] = csub(t0, t2);
      dl[od + 3 * Ns] = csub(t1, t3);
    } else if constexpr (R == 3) {
      double2 a0 = sl[j], a1 = sl[j + nb], a2 = sl[j + 2 * nb];
      if constexpr (Ns > 1) {
        double2 w1 = tw[k * tstride], w2 = tw[2 * k * tstride];
        if (INV) { w1 = cconj(w1); w2 = cconj(w2); }
        a1 = cmul(a1, w1); a2 = cmul(a2, w2);
      }
      double2 t = cadd(a1, a2), d = csub(a1, a2);
      double2 m = make_double2(a0.x - 0.5 * t.x, a0.y - 0.5 * t.y);
      const double sd = INV ? -CORAL_SIN60 : CORAL_SIN60;
      double2 isd = make_double2(-sd * d.y, sd * d.x);
      dl[od] = cadd(a0, t);
      dl[od + Ns] = csub(m, isd);
      dl[od + 2 * Ns] = cadd(m, isd);
    } else {
      double2 a0 = sl[j], a1 = sl[j + nb];
      if constexpr (Ns > 1) {
        double2 w1 = tw[k * tstride];
        if (INV) w1 = cconj(w1);
        a1 = cmul(a1, w1);
      }
      dl[od] = cadd(a0, a1);
      dl[od + Ns] = csub(a0, a1);
    }
  }
}

template <int N, int S, int Ns, bool INV>
__device__ __forceinline__ double2* fft_stages_t(double2* src, double2* dst, int nl, const double2* tw) {
  constexpr PlanC P = make_planc(N);
  if constexpr (S >= P.nst) {
    return src;
  } else {
    constexpr int R = P.r[S];
    fft_stage_t<N, R, Ns, INV>(src, dst, nl, tw);
    __syncthreads();
    return fft_stages_t<N, S + 1, Ns * R, INV>(dst, src, nl, tw);
  }
}

// Batched FFT with a compile-time length NC, or the runtime plan when NC == 0.
template <int NC, bool INV>
__device__ __forceinline__ double2* fft_lines_n(double2* A, double2* B, int nl, const FftPlan& p) {
  if constexpr (NC == 0) {
    return fft_lines<INV>(A, B, nl, p);
  } else {
    static_assert(make_planc(NC).nst > 0, "transform length must be 2^a 3^b");
    return fft_stages_t<NC, 0, 1, INV>(A, B, nl, p.tw);
  }
}

}  // namespace coral
