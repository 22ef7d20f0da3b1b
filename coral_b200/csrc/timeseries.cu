// Timeseries reduction: the per-CTA partial sums of the timeseries objects
// (volume averages and horizontal averages at grid levels, computed by the z
// kernels on the first stage's physical fields) totalled over the grid, as
// output_global_quantities does with its loops over the local grid
// (src/plane_layer/PL_IMEX_timestepping_output.f90:30-127).
#include "device.hpp"

namespace coral {
namespace {

constexpr int kTsThreads = 256;

// one CTA per object; each thread sums a fixed strided subset, then a fixed
// tree: the result does not depend on scheduling
__global__ void __launch_bounds__(kTsThreads) k_ts_reduce(const double* part, size_t ncta, double scale,
                                                          double* out) {
  __shared__ double red[kTsThreads];
  const int o = blockIdx.x;
  double s = 0.0;
  for (size_t c = threadIdx.x; c < ncta; c += kTsThreads) s += part[c * kMaxTs + o];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = kTsThreads / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[o] = red[0] * scale;
}

}  // namespace

void launch_ts_reduce(const double* part, size_t ncta, int nobj, double scale, double* out, cudaStream_t s) {
  if (nobj <= 0) return;
  k_ts_reduce<<<nobj, kTsThreads, 0, s>>>(part, ncta, scale, out);
}

}  // namespace coral

namespace coral {
namespace {

// The kx = 0 line of a coupled state onto its Hermitian part:
// f(0, ky) <- (f(0, ky) + conj f(0, -ky)) / 2 and f(0, -ky) <- its conjugate;
// the self-conjugate ky = 0 and Nyquist entries keep their real parts.  A real
// physical field has a Hermitian kx = 0 line; the anti-Hermitian part is
// invisible to the inverse transform (the x c2r keeps only the real part of the
// kx = 0 coefficient), so nothing in the time step feeds back on it, and where
// the linear operator of its (kx = 0, ky) system is unstable it grows without
// bound until round-off carries it into the physical fields.  The projection
// removes exactly that part and leaves every physical value unchanged.
__global__ void k_hermitian_kx0(double2* field, int NYA, int T) {
  const int half = NYA / 2;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < (half + 1) * T; e += gridDim.x * blockDim.x) {
    const int iy = e / T, t = e - iy * T;
    if (iy == 0 || (iy == half && NYA % 2 == 0)) {
      double2& a = field[(size_t)iy * T + t];
      a.y = 0.0;
      continue;
    }
    double2& a = field[(size_t)iy * T + t];
    double2& b = field[(size_t)(NYA - iy) * T + t];
    const double2 h = make_double2(0.5 * (a.x + b.x), 0.5 * (a.y - b.y));
    a = h;
    b = make_double2(h.x, -h.y);
  }
}

}  // namespace

void launch_hermitian_kx0(double2* field, int NYA, int T, cudaStream_t s) {
  const int n = (NYA / 2 + 1) * T;
  k_hermitian_kx0<<<(n + 255) / 256, 256, 0, s>>>(field, NYA, T);
}

}  // namespace coral
