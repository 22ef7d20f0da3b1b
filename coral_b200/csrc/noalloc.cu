// Inverse transform (spectral -> physical) of one scalar field that allocates
// no device memory.
//
// Some callers cannot call cudaMalloc: a Fortran code whose device memory is
// owned by another runtime or pool allocator, a plugin running inside a host
// application that forbids allocations after start-up, or work recorded while
// an allocator is frozen.  They pass their own input and output buffers; the
// two intermediate arrays of the transform (after the y pass and after the x
// pass) live in the file-scope __device__ array below, which every GPU that
// loads this library holds until the process exits.
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/coral_b200.h"
#include "device.hpp"
#include "host.hpp"

using namespace coral;

namespace {

constexpr size_t kScratchBytes = size_t(64) << 20;  // 64 MiB, the stated maximum
__device__ __align__(256) unsigned char g_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mutex;
void* g_scratch_addr[kMaxDevices] = {};

// Device address of g_scratch on the current device, looked up once per device
// (the array's name in host code is only a stand-in for the symbol).
void* scratch_address() {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) throw CoralError(CORAL_ENODEV, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) throw CoralError(CORAL_EBADARG, "device index beyond the supported range");
  std::lock_guard<std::mutex> lock(g_mutex);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_scratch);
    if (e != cudaSuccess || !p)
      throw CoralError(CORAL_ECUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
    g_scratch_addr[dev] = p;
  }
  return g_scratch_addr[dev];
}

// exp(-i pi k * f / N) for k < N, from sincospi: f = 2 gives the FFT twiddles,
// f = 1/2 the pre/post-rotation of the FFT-based Chebyshev transform
__global__ void k_twiddles(double2* tw, int N, double f) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < N; k += gridDim.x * blockDim.x) {
    double s, c;
    sincospi(-f * (double)k / (double)N, &s, &c);
    tw[k] = make_double2(c, s);
  }
}

bool smooth23(int n) {
  if (n <= 0) return false;
  while (n % 2 == 0) n /= 2;
  while (n % 3 == 0) n /= 3;
  return n == 1;
}

FftPlan plan_in(int N, double2* tw) {
  FftPlan p{};
  p.N = N;
  int n = N, s = 0;
  while (n % 4 == 0) { p.radix[s++] = 4; n /= 4; }
  while (n % 3 == 0) { p.radix[s++] = 3; n /= 3; }
  while (n % 2 == 0) { p.radix[s++] = 2; n /= 2; }
  p.nst = s;
  p.tw = tw;
  return p;
}

size_t up256(size_t b) { return (b + 255) & ~size_t(255); }

}  // namespace

extern "C" int coral_spec_to_phys_noalloc(int NX, int NY, int NZ, const double* spec, double* phys, void* stream) {
  try {
    if (!spec || !phys) throw CoralError(CORAL_EBADARG, "coral_spec_to_phys_noalloc: null buffer");
    if (NX <= 0 || NY <= 0 || NZ <= 0 || NX % 4 || NY % 4 || NZ % 4)
      throw CoralError(CORAL_EBADARG, "coral_spec_to_phys_noalloc: NX, NY, NZ must be positive multiples of 4");
    const int NXA = 3 * NX / 2, NYA = 3 * NY / 2, NZA = 3 * NZ / 2, NXH = NX / 2;
    if (!smooth23(NXA) || !smooth23(NYA) || !smooth23(NZA))
      throw CoralError(CORAL_EBADARG, "coral_spec_to_phys_noalloc: grid sizes must be of the form 2^a 3^b");
    // scratch layout: three twiddle tables, then the two intermediate arrays
    const size_t o_ty = 0;
    const size_t o_tx = o_ty + up256((size_t)NYA * sizeof(double2));
    const size_t o_tz = o_tx + up256((size_t)NXA * sizeof(double2));
    const size_t o_td = o_tz + up256((size_t)NZA * sizeof(double2));
    const size_t o_y1 = o_td + up256((size_t)NZA * sizeof(double2));
    const size_t o_y2 = o_y1 + up256((size_t)NYA * NXH * NZ * sizeof(double2));
    const size_t need = o_y2 + up256((size_t)NYA * NXA * NZ * sizeof(double));
    if (need > kScratchBytes)
      throw CoralError(CORAL_EBADARG, "coral_spec_to_phys_noalloc: grid needs " + std::to_string(need) +
                                          " bytes of scratch, above the built-in maximum of " +
                                          std::to_string(kScratchBytes) + " bytes (64 MiB)");
    unsigned char* base = static_cast<unsigned char*>(scratch_address());
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    double2* ty = reinterpret_cast<double2*>(base + o_ty);
    double2* tx = reinterpret_cast<double2*>(base + o_tx);
    double2* tz = reinterpret_cast<double2*>(base + o_tz);
    double2* td = reinterpret_cast<double2*>(base + o_td);
    double2* Y1 = reinterpret_cast<double2*>(base + o_y1);
    double* Y2 = reinterpret_cast<double*>(base + o_y2);
    // every scratch byte that is read is written first in this call (twiddles,
    // then the y pass fills Y1, the x pass fills Y2), so nothing needs clearing
    k_twiddles<<<8, 128, 0, s>>>(ty, NYA, 2.0);
    k_twiddles<<<8, 128, 0, s>>>(tx, NXA, 2.0);
    k_twiddles<<<8, 128, 0, s>>>(tz, NZA, 2.0);
    k_twiddles<<<8, 128, 0, s>>>(td, NZA, 0.5);
    const Dims d{NXH, NYA, NXA, NZ, NZA};
    const FftPlan py = plan_in(NYA, ty), px = plan_in(NXA, tx), pz = plan_in(NZA, tz);
    launch_inv_y(d, 1, nullptr, StateSet{}, reinterpret_cast<const double2*>(spec), nullptr, nullptr, Y1, py, s);
    launch_inv_x(d, 1, Y1, Y2, px, s);
    launch_inv_z(d, 1, Y2, phys, pz, td, nullptr, nullptr, s);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) throw CoralError(CORAL_ECUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
    return CORAL_OK;
  } catch (const CoralError& err) {
    set_global_error(err.what());
    return err.code;
  }
}
