// Learned subgrid closure: a small stencil network that predicts, on a coarse
// grid, the subgrid part of every quadratic variable,
//   tau_q = P(q_fine) - q(P(fields_fine))        (P: truncation to the coarse modes),
// from the resolved full variables.  Inside the time step its outputs are added
// to the pointwise products before their forward transform, so they reach the
// explicit nonlinear term K_hat through the recipe's own NL operator (the
// divergence and quasi-inverse integration of the subgrid fluxes).  The
// reference has no learned closure; its nonlinear terms are the products of
// src/plane_layer/PL_IMEX_timestepping_marching.f90:279-352.
//
// Network (every grid point independently):
//   x  = 5 channels (u, v, w, T scaled by in_scale, and the wall-normal
//        coordinate z' in [-1, 1]) at the 27 points of the 3 x 3 x 3 stencil
//        (periodic in x and y, zero beyond the walls): 135 inputs
//   h1 = tanh(W0 x + b0)      64
//   h2 = tanh(W1 h1 + b1)     64
//   h3 = tanh(W2 h2 + b2)     64
//   y  = W3 h3 + b3           9 outputs, tau_q = out_scale[q] y_q
// Weights are used in BF16 (FP32 master copies for the optimiser), biases,
// activations and every accumulation in FP32.  Forward, backward (loss = mean
// over points of sum_q (y_q - target_q / out_scale[q])^2) and Adam are the
// kernels below; one CTA takes 128 points and keeps their inputs, activations
// and deltas in shared memory (feature-major, so a thread's column is
// conflict-free), the weights in BF16 in shared memory (broadcast reads).
#include <cuda_bf16.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/coral_b200.h"
#include "device.hpp"
#include "host.hpp"

namespace coral {
namespace {

constexpr int kCin = 5, kTaps = 27, kIn = kCin * kTaps, kHid = 64, kOut = 9;
constexpr int kP = 128;  // points per CTA (threads)
constexpr int kR = kP + 1;  // row stride of the feature-major arrays: a column read by all threads is
                            // conflict-free, and so is a row read by all threads (the weight-gradient sums)
// flat parameter layout: W0 [kHid][kIn], b0, W1 [kHid][kHid], b1, W2 [kHid][kHid], b2, W3 [kOut][kHid], b3
constexpr int oW0 = 0, oB0 = oW0 + kHid * kIn, oW1 = oB0 + kHid, oB1 = oW1 + kHid * kHid, oW2 = oB1 + kHid,
              oB2 = oW2 + kHid * kHid, oW3 = oB2 + kHid, oB3 = oW3 + kOut * kHid, kNParam = oB3 + kOut;

struct NetDev {
  const __nv_bfloat16* w16;  // kNParam (biases too, unused in BF16)
  const float* w32;          // master copies (the biases are read from here)
  float in_scale[4], out_scale[kOut];
};

// shared-memory layout of a CTA (floats unless noted)
constexpr size_t sX = (size_t)kIn * kR, sH = (size_t)kHid * kR;
constexpr size_t kSmemFloats = sX + 3 * sH + (size_t)kOut * kR;
constexpr size_t kSmemBytes = kSmemFloats * sizeof(float) + (size_t)kNParam * sizeof(__nv_bfloat16) + 16;

__device__ __forceinline__ float bf(const __nv_bfloat16* w, int i) { return __bfloat162float(w[i]); }

// Gather the 135 inputs of point (y, x, z) of a grid (NYA, NXA, NZA) into column
// t of X; fields: 4 arrays [y][x][z] (double or float)
template <typename F>
__device__ __forceinline__ void gather(float* X, int t, const F* f0, const F* f1, const F* f2, const F* f3,
                                       int NYA, int NXA, int NZA, int y, int x, int z, const float* in_scale,
                                       const double* zeta) {
  const F* fs[4] = {f0, f1, f2, f3};
  int tap = 0;
  for (int dy = -1; dy <= 1; ++dy)
    for (int dx = -1; dx <= 1; ++dx)
      for (int dz = -1; dz <= 1; ++dz, ++tap) {
        const int yy = (y + dy + NYA) % NYA, xx = (x + dx + NXA) % NXA, zz = z + dz;
        const bool in = zz >= 0 && zz < NZA;
        const size_t lin = ((size_t)yy * NXA + xx) * NZA + (in ? zz : 0);
#pragma unroll
        for (int c = 0; c < 4; ++c) X[(c * kTaps + tap) * kR + t] = in ? (float)fs[c][lin] * in_scale[c] : 0.0f;
        X[(4 * kTaps + tap) * kR + t] = in ? (float)zeta[zz] : 0.0f;
      }
}

// dense layer on the columns of the CTA: out[o][t] = act(b[o] + sum_i W[o][i] in[i][t])
template <int NI, int NO, bool TANH>
__device__ __forceinline__ void layer(const float* in, float* out, const __nv_bfloat16* W, const float* b, int t) {
  for (int o0 = 0; o0 < NO; o0 += 4) {
    float acc[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[j] = (o0 + j < NO) ? b[o0 + j] : 0.0f;
    for (int i = 0; i < NI; ++i) {
      const float xv = in[i * kR + t];
#pragma unroll
      for (int j = 0; j < 4; ++j)
        if (o0 + j < NO) acc[j] = fmaf(bf(W, (o0 + j) * NI + i), xv, acc[j]);
    }
#pragma unroll
    for (int j = 0; j < 4; ++j)
      if (o0 + j < NO) out[(o0 + j) * kR + t] = TANH ? tanhf(acc[j]) : acc[j];
  }
}

// Forward of kP points per CTA.  Inference (targets == null): point p is grid
// point p (linear [y][x][z]) of fields (double), tau_q written (double) to
// out[q][p] * out_scale[q].  Training (targets non-null): point p is
// points[p] = snapshot * npoint + linear index, inputs / targets from the
// float dataset; the loss and its gradient are accumulated (grad, loss).
template <bool TRAIN, typename F>
__global__ void __launch_bounds__(kP, 1) k_closure(NetDev net, const F* fields, long long snap_stride, int NYA, int NXA,
                                                  int NZA, const double* zeta, const long long* points, long long npts,
                                                  const float* targets, double* tau, float* grad, double* loss) {
  extern __shared__ __align__(16) float smem[];
  float* X = smem;
  float* H1 = X + sX;
  float* H2 = H1 + sH;
  float* H3 = H2 + sH;
  float* Y = H3 + sH;
  __nv_bfloat16* W = reinterpret_cast<__nv_bfloat16*>(Y + (size_t)kOut * kR);
  const int t = threadIdx.x;
  for (int i = t; i < kNParam; i += kP) W[i] = net.w16[i];
  const long long p = (long long)blockIdx.x * kP + t;
  const long long npoint = (long long)NYA * NXA * NZA;
  const bool ok = p < npts;
  long long snap = 0, lin = ok ? p : 0;
  if (TRAIN && ok) {
    const long long g = points[p];
    snap = g / npoint;
    lin = g - snap * npoint;
  }
  const int z = (int)(lin % NZA), x = (int)((lin / NZA) % NXA), y = (int)(lin / ((long long)NZA * NXA));
  const F* base = fields + snap * snap_stride;
  gather(X, t, base, base + npoint, base + 2 * npoint, base + 3 * npoint, NYA, NXA, NZA, y, x, z, net.in_scale, zeta);
  __syncthreads();
  layer<kIn, kHid, true>(X, H1, W + oW0, net.w32 + oB0, t);
  layer<kHid, kHid, true>(H1, H2, W + oW1, net.w32 + oB1, t);
  layer<kHid, kHid, true>(H2, H3, W + oW2, net.w32 + oB2, t);
  layer<kHid, kOut, false>(H3, Y, W + oW3, net.w32 + oB3, t);
  if (!TRAIN) {
    if (ok)
      for (int q = 0; q < kOut; ++q) tau[(size_t)q * npoint + lin] = (double)(Y[q * kR + t] * net.out_scale[q]);
    return;
  }
  // ---- loss and its gradient with respect to y (the mean over all npts points) ----
  __shared__ float red[kP / 32];
  float l = 0.0f;
  const float inv = 1.0f / (float)npts;
  for (int q = 0; q < kOut; ++q) {
    float d = 0.0f;
    if (ok) {
      const float tg = targets[snap * (long long)kOut * npoint + (long long)q * npoint + lin] / net.out_scale[q];
      d = Y[q * kR + t] - tg;
    }
    l += d * d;
    Y[q * kR + t] = 2.0f * d * inv;  // dL/dy
  }
  for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
  if ((t & 31) == 0) red[t >> 5] = l;
  __syncthreads();
  if (t == 0) {
    float s = 0.0f;
    for (int w = 0; w < kP / 32; ++w) s += red[w];
    atomicAdd(loss, (double)s * inv);
  }
  // ---- backward: weight gradients summed over the CTA's points, then atomics ----
  // dW3[o][i] = sum_t dy[o][t] h3[i][t]; db3[o] = sum_t dy[o][t]
  auto wgrad = [&](const float* dOut, const float* In, int NO, int NI, int oW, int oB) {
    for (int e = t; e < NO * NI; e += kP) {
      const int o = e / NI, i = e - o * NI;
      float s = 0.0f;
      for (int tt = 0; tt < kP; ++tt) s = fmaf(dOut[o * kR + tt], In[i * kR + tt], s);
      atomicAdd(grad + oW + e, s);
    }
    for (int o = t; o < NO; o += kP) {
      float s = 0.0f;
      for (int tt = 0; tt < kP; ++tt) s += dOut[o * kR + tt];
      atomicAdd(grad + oB + o, s);
    }
  };
  // delta of a tanh layer in place: dIn[i][t] = (sum_o W[o][i] dOut[o][t]) (1 - h[i][t]^2)
  auto backprop = [&](const float* dOut, float* Hin, const __nv_bfloat16* Wl, int NO) {
    float dv[kHid];
#pragma unroll
    for (int i = 0; i < kHid; ++i) dv[i] = 0.0f;
    for (int o = 0; o < NO; ++o) {
      const float g = dOut[o * kR + t];
#pragma unroll
      for (int i = 0; i < kHid; ++i) dv[i] = fmaf(bf(Wl, o * kHid + i), g, dv[i]);
    }
#pragma unroll
    for (int i = 0; i < kHid; ++i) {
      const float h = Hin[i * kR + t];
      Hin[i * kR + t] = dv[i] * (1.0f - h * h);
    }
  };
  __syncthreads();
  wgrad(Y, H3, kOut, kHid, oW3, oB3);
  __syncthreads();
  backprop(Y, H3, W + oW3, kOut);  // H3 <- delta3
  __syncthreads();
  wgrad(H3, H2, kHid, kHid, oW2, oB2);
  __syncthreads();
  backprop(H3, H2, W + oW2, kHid);  // H2 <- delta2
  __syncthreads();
  wgrad(H2, H1, kHid, kHid, oW1, oB1);
  __syncthreads();
  backprop(H2, H1, W + oW1, kHid);  // H1 <- delta1
  __syncthreads();
  wgrad(H1, X, kHid, kIn, oW0, oB0);
}

// Adam (Kingma & Ba, 2015) on the FP32 master parameters; the BF16 copies are
// refreshed and the gradient cleared
__global__ void k_adam(float* w32, __nv_bfloat16* w16, float* g, float* m, float* v, int n, float lr, float b1,
                       float b2, float eps, float c1, float c2) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float wi = w32[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    w32[i] = wi;
    w16[i] = __float2bfloat16(wi);
    g[i] = 0.0f;
  }
}

__global__ void k_to_bf16(const float* w32, __nv_bfloat16* w16, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    w16[i] = __float2bfloat16(w32[i]);
}

}  // namespace

// ---- the network object ----------------------------------------------------------------
struct ClosureImpl {
  int device = 0;
  float *w32 = nullptr, *g = nullptr, *m = nullptr, *v = nullptr;
  __nv_bfloat16* w16 = nullptr;
  double* loss = nullptr;
  double* zeta = nullptr;
  int zeta_n = 0;
  float in_scale[4] = {1, 1, 1, 1}, out_scale[kOut] = {1, 1, 1, 1, 1, 1, 1, 1, 1};
  long long adam_t = 0;
  std::string err;
};

size_t closure_param_count() { return kNParam; }

NetDev net_dev(const ClosureImpl* c) {
  NetDev n{};
  n.w16 = c->w16;
  n.w32 = c->w32;
  for (int i = 0; i < 4; ++i) n.in_scale[i] = c->in_scale[i];
  for (int i = 0; i < kOut; ++i) n.out_scale[i] = c->out_scale[i];
  return n;
}

void closure_set_smem() {
  static bool done = false;
  if (done) return;
  cudaFuncSetAttribute(k_closure<false, double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemBytes);
  cudaFuncSetAttribute(k_closure<true, float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemBytes);
  done = true;
}

// z' = (z - center) / (gap / 2) of the Gauss-Chebyshev grid, uploaded once per size
void closure_zeta(ClosureImpl* c, int NZA) {
  if (c->zeta && c->zeta_n == NZA) return;
  if (c->zeta) cudaFree(c->zeta);
  std::vector<double> z(NZA);
  const long double pi = 3.141592653589793238462643383279502884L;
  for (int i = 0; i < NZA; ++i) z[i] = (double)cosl(pi * (2.0L * (i + 1) - 1.0L) / (2.0L * NZA));
  if (cudaMalloc(&c->zeta, NZA * sizeof(double)) != cudaSuccess) throw CoralError(CORAL_ENOMEM, "closure: zeta");
  cudaMemcpy(c->zeta, z.data(), NZA * sizeof(double), cudaMemcpyHostToDevice);
  c->zeta_n = NZA;
}

// inference on a whole grid: 4 full-variable fields [f][y][x][z] (double) -> tau [9][y][x][z]
void closure_infer(ClosureImpl* c, const double* fields, int NYA, int NXA, int NZA, double* tau, cudaStream_t s) {
  closure_set_smem();
  closure_zeta(c, NZA);
  const long long np = (long long)NYA * NXA * NZA;
  k_closure<false, double><<<(unsigned)((np + kP - 1) / kP), kP, kSmemBytes, s>>>(
      net_dev(c), fields, 0, NYA, NXA, NZA, c->zeta, nullptr, np, nullptr, tau, nullptr, nullptr);
}

}  // namespace coral

using namespace coral;

struct coral_closure : ClosureImpl {};

namespace {

thread_local std::string g_closure_error;

template <typename F>
int cguard(coral_closure* c, F&& f) {
  if (!c) return CORAL_EBADARG;
  try {
    if (cudaSetDevice(c->device) != cudaSuccess) throw CoralError(CORAL_ECUDA, "cudaSetDevice");
    f();
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) throw CoralError(CORAL_ECUDA, std::string("closure kernel: ") + cudaGetErrorString(e));
    return CORAL_OK;
  } catch (const CoralError& x) {
    c->err = x.what();
    return x.code;
  }
}

}  // namespace

namespace coral {
ClosureImpl* closure_impl(coral_closure* c) { return c; }
}  // namespace coral

extern "C" {

int coral_closure_create(int device, unsigned long long seed, coral_closure** out) {
  if (!out) return CORAL_EBADARG;
  *out = nullptr;
  auto* c = new coral_closure();
  c->device = device;
  if (cudaSetDevice(device) != cudaSuccess) {
    g_closure_error = "closure: no such device";
    delete c;
    return CORAL_ENODEV;
  }
  const size_t n = kNParam;
  bool okm = cudaMalloc(&c->w32, n * 4) == cudaSuccess && cudaMalloc(&c->g, n * 4) == cudaSuccess &&
             cudaMalloc(&c->m, n * 4) == cudaSuccess && cudaMalloc(&c->v, n * 4) == cudaSuccess &&
             cudaMalloc(&c->w16, n * 2) == cudaSuccess && cudaMalloc(&c->loss, 8) == cudaSuccess;
  if (!okm) {
    g_closure_error = "closure: device allocation failed";
    coral_closure_destroy(c);
    return CORAL_ENOMEM;
  }
  // Glorot-uniform weights from a 64-bit LCG (Knuth's MMIX constants), zero biases
  std::vector<float> w(n, 0.0f);
  unsigned long long st = seed * 6364136223846793005ull + 1442695040888963407ull;
  auto uni = [&]() {
    st = st * 6364136223846793005ull + 1442695040888963407ull;
    return (double)(st >> 11) * (1.0 / 9007199254740992.0);
  };
  auto fill = [&](int off, int no, int ni) {
    const double a = std::sqrt(6.0 / (double)(no + ni));
    for (int i = 0; i < no * ni; ++i) w[off + i] = (float)((2.0 * uni() - 1.0) * a);
  };
  fill(oW0, kHid, kIn);
  fill(oW1, kHid, kHid);
  fill(oW2, kHid, kHid);
  fill(oW3, kOut, kHid);
  cudaMemcpy(c->w32, w.data(), n * 4, cudaMemcpyHostToDevice);
  cudaMemset(c->g, 0, n * 4);
  cudaMemset(c->m, 0, n * 4);
  cudaMemset(c->v, 0, n * 4);
  k_to_bf16<<<64, 256>>>(c->w32, c->w16, (int)n);
  if (cudaDeviceSynchronize() != cudaSuccess) {
    g_closure_error = "closure: initialisation failed";
    coral_closure_destroy(c);
    return CORAL_ECUDA;
  }
  *out = c;
  return CORAL_OK;
}

void coral_closure_destroy(coral_closure* c) {
  if (!c) return;
  cudaSetDevice(c->device);
  cudaFree(c->w32);
  cudaFree(c->g);
  cudaFree(c->m);
  cudaFree(c->v);
  cudaFree(c->w16);
  cudaFree(c->loss);
  if (c->zeta) cudaFree(c->zeta);
  delete c;
}

const char* coral_closure_last_error(const coral_closure* c) { return c ? c->err.c_str() : g_closure_error.c_str(); }

int coral_closure_param_count(void) { return kNParam; }

int coral_closure_set_scales(coral_closure* c, const float* in_scale4, const float* out_scale9) {
  return cguard(c, [&] {
    if (!in_scale4 || !out_scale9) throw CoralError(CORAL_EBADARG, "null scales");
    for (int i = 0; i < 4; ++i) c->in_scale[i] = in_scale4[i];
    for (int i = 0; i < kOut; ++i) {
      if (!(out_scale9[i] > 0.0f)) throw CoralError(CORAL_EBADARG, "output scales must be > 0");
      c->out_scale[i] = out_scale9[i];
    }
  });
}

int coral_closure_get_params(coral_closure* c, float* params, int n) {
  return cguard(c, [&] {
    if (!params || n < kNParam) throw CoralError(CORAL_EBADARG, "buffer smaller than the parameter count");
    if (cudaMemcpy(params, c->w32, kNParam * 4, cudaMemcpyDeviceToHost) != cudaSuccess)
      throw CoralError(CORAL_ECUDA, "copy");
  });
}

int coral_closure_set_params(coral_closure* c, const float* params, int n) {
  return cguard(c, [&] {
    if (!params || n < kNParam) throw CoralError(CORAL_EBADARG, "buffer smaller than the parameter count");
    if (cudaMemcpy(c->w32, params, kNParam * 4, cudaMemcpyHostToDevice) != cudaSuccess)
      throw CoralError(CORAL_ECUDA, "copy");
    k_to_bf16<<<64, 256>>>(c->w32, c->w16, kNParam);
    cudaDeviceSynchronize();
  });
}

int coral_closure_get_gradient(coral_closure* c, float* grad, int n) {
  return cguard(c, [&] {
    if (!grad || n < kNParam) throw CoralError(CORAL_EBADARG, "buffer smaller than the parameter count");
    if (cudaMemcpy(grad, c->g, kNParam * 4, cudaMemcpyDeviceToHost) != cudaSuccess)
      throw CoralError(CORAL_ECUDA, "copy");
  });
}

int coral_closure_train(coral_closure* c, const float* inputs, const float* targets, int nsnap, int NXA, int NYA,
                        int NZA, const long long* points, long long npts, float lr, int apply, double* loss) {
  return cguard(c, [&] {
    if (!inputs || !targets || !points || npts <= 0 || nsnap <= 0 || NXA <= 0 || NYA <= 0 || NZA <= 0)
      throw CoralError(CORAL_EBADARG, "closure_train: bad arguments");
    closure_set_smem();
    closure_zeta(c, NZA);
    const long long np = (long long)NYA * NXA * NZA;
    cudaMemset(c->loss, 0, 8);
    k_closure<true, float><<<(unsigned)((npts + kP - 1) / kP), kP, kSmemBytes>>>(
        net_dev(c), inputs, 4 * np, NYA, NXA, NZA, c->zeta, points, npts, targets, nullptr, c->g, c->loss);
    if (apply) {
      ++c->adam_t;
      const float b1 = 0.9f, b2 = 0.999f;
      k_adam<<<64, 256>>>(c->w32, c->w16, c->g, c->m, c->v, kNParam, lr, b1, b2, 1e-8f,
                          1.0f - std::pow(b1, (float)c->adam_t), 1.0f - std::pow(b2, (float)c->adam_t));
    }
    double l = 0.0;
    if (cudaMemcpy(&l, c->loss, 8, cudaMemcpyDeviceToHost) != cudaSuccess) throw CoralError(CORAL_ECUDA, "loss");
    if (loss) *loss = l;
  });
}

int coral_closure_zero_gradient(coral_closure* c) {
  return cguard(c, [&] { cudaMemset(c->g, 0, kNParam * 4); });
}

int coral_closure_infer(coral_closure* c, const double* fields, int NXA, int NYA, int NZA, double* tau, void* stream) {
  return cguard(c, [&] {
    if (!fields || !tau) throw CoralError(CORAL_EBADARG, "null buffer");
    closure_infer(c, fields, NYA, NXA, NZA, tau, static_cast<cudaStream_t>(stream));
  });
}

}  // extern "C"
