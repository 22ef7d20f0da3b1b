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
constexpr int kMaxModes = 1 << 16;                  // per direction, checked first
__device__ __align__(256) unsigned char g_scratch[kScratchBytes];

// The device address of g_scratch, looked up once per device and CUDA context
// with that device current (in host code the array's name is only a stand-in
// for the symbol, not a device address).  The cache is keyed by the context's
// unique id, so a cudaDeviceReset in the caller's process (a new primary
// context, the module loaded again) triggers a fresh lookup.
struct ScratchSlot {
  unsigned long long ctx_id = 0;
  void* addr = nullptr;
};
constexpr int kMaxDevices = 64;
std::mutex g_mutex;
ScratchSlot g_slot[kMaxDevices];

typedef int (*CtxGetCurrentFn)(void**);
typedef int (*CtxGetIdFn)(void*, unsigned long long*);

// id of the current CUDA context (0 if the driver cannot tell); the driver's
// entry points are fetched through the runtime, so the library needs no link
// against libcuda
unsigned long long current_context_id() {
  static CtxGetCurrentFn get_cur = nullptr;
  static CtxGetIdFn get_id = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    cudaDriverEntryPointQueryResult q1, q2;
    void* f1 = nullptr;
    void* f2 = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f1, cudaEnableDefault, &q1) == cudaSuccess &&
        q1 == cudaDriverEntryPointSuccess &&
        cudaGetDriverEntryPoint("cuCtxGetId", &f2, cudaEnableDefault, &q2) == cudaSuccess &&
        q2 == cudaDriverEntryPointSuccess) {
      get_cur = reinterpret_cast<CtxGetCurrentFn>(f1);
      get_id = reinterpret_cast<CtxGetIdFn>(f2);
    }
  }
  if (!get_cur || !get_id) return 0;
  void* ctx = nullptr;
  unsigned long long id = 0;
  if (get_cur(&ctx) != 0 || !ctx || get_id(ctx, &id) != 0) return 0;
  return id;
}

void* scratch_address() {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) throw CoralError(CORAL_ENODEV, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) throw CoralError(CORAL_EBADARG, "device index beyond the supported range");
  // before the runtime has made the device's context current the id reads 0,
  // which always triggers a lookup (cudaGetSymbolAddress creates the context)
  const unsigned long long ctx = current_context_id();
  std::lock_guard<std::mutex> lock(g_mutex);
  ScratchSlot& slot = g_slot[dev];
  if (!slot.addr || slot.ctx_id != ctx || ctx == 0) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_scratch);
    if (e != cudaSuccess || !p)
      throw CoralError(CORAL_ECUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
    slot.addr = p;
    slot.ctx_id = ctx;
  }
  return slot.addr;
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
    // sizes are checked before any arithmetic on them (3 N / 2 must not overflow)
    if (NX <= 0 || NY <= 0 || NZ <= 0 || NX > kMaxModes || NY > kMaxModes || NZ > kMaxModes || NX % 4 || NY % 4 ||
        NZ % 4)
      throw CoralError(CORAL_EBADARG, "coral_spec_to_phys_noalloc: NX, NY, NZ must be multiples of 4 in [4, " +
                                          std::to_string(kMaxModes) + "]");
    // an error left pending by earlier, unrelated work is not this call's: it is
    // reported as such and left in place for its owner
    const cudaError_t pending = cudaPeekAtLastError();
    if (pending != cudaSuccess)
      throw CoralError(CORAL_ECUDA, std::string("coral_spec_to_phys_noalloc: a CUDA error was already pending "
                                                "before the call: ") + cudaGetErrorString(pending));
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
    // nothing was pending at entry, so an error now comes from these launches
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) throw CoralError(CORAL_ECUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
    return CORAL_OK;
  } catch (const CoralError& err) {
    set_global_error(err.what());
    return err.code;
  }
}
