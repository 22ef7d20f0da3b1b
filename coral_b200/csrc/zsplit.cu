// Split-precision z (Chebyshev) transforms on the 5th-generation tensor cores.
//
// The z passes of a stage -- the REDFT01 of the full variables
// (src/slabs.fftw3mpi/transforms.f90:216-223) and the REDFT10 of the quadratic
// variables (:243-249), with the pointwise products between them
// (src/plane_layer/PL_IMEX_timestepping_marching.f90:279-291) -- run here as
// dense contractions over the Chebyshev / grid index, one column (x, y) at a
// time:
//   inverse  phys[col][z] = sum_n Cinv[z][n] Y2[col][n],  Cinv = (n ? 2 : 1) cos(pi n (2z+1) / 2NZAA)
//   forward  Q2[col][n]   = sum_z Cfwd[n][z] q[col][z],   Cfwd = 2 cos(pi n (2z+1) / 2NZAA)
// with the operands split into integer digits (an Ozaki-type scheme): a data
// value v of a column whose largest magnitude is below 2^e becomes
// m = rint(v 2^(38-e)), |m| <= 2^38, written in five signed base-256 digits
// m = d0 2^32 + d1 2^24 + d2 2^16 + d3 2^8 + d4 (the lower four centred in
// [-128, 127], |d0| <= 64); a matrix entry c (|c| <= 2) becomes rint(c 2^36)
// in the same digits.  Centred digits make the neglected low-order products
// random in sign: with unsigned digits they all add with one sign and their
// bias grows with K.  The digit products with i + j <= 4 (15 of them) run as
// tcgen05.mma kind::i8 (s8 x s8) with INT32 accumulators in tensor memory, one
// accumulator per anti-diagonal d = i + j; the accumulation is exact (each
// anti-diagonal sum stays below 2^25 for K <= 288).  The epilogue combines the
// five accumulators exactly in 64-bit integers, S = sum_d D_d 2^(32-8d), and
// converts once to FP64: out = S 2^(e-42).  The result is good to about
// 3e-11 relative L2 (1e-9 of a column's largest value at worst) for K = 192 /
// 288, against ~1e-16 for the FP64 transforms.
//
// Kernel shape (one CTA per SM: 215 KB of shared memory, 512 TMEM columns):
// a CTA takes 128 columns of one variable (the MMA's M), slices the whole
// column range of K into shared memory once (5 digit planes in the K-major
// canonical layout without swizzle), then for each tile of 96 outputs (the
// MMA's N; 3 tiles for 288 outputs, 2 for 192) streams the matrix digits of
// one K step (32) at a time through a double buffer and issues the 15 MMAs of
// that step from one thread; the step's tcgen05.commit releases its buffer.
// The epilogue reads the accumulators with tcgen05.ld (thread = column) and
// writes each column's outputs contiguously.  Every wait on an mbarrier is
// bounded: on a timeout the kernel sets bit 1 of the handle's flag word,
// releases its tensor memory and returns.
#include <cstdint>
#include <vector>

#include "../../include/coral_b200.h"
#include "device.hpp"
#include "host.hpp"

namespace coral {
namespace {

constexpr int kS = 5;         // digit planes
constexpr int kM = 128;       // columns per CTA (MMA M)
constexpr int kN = 96;        // outputs per tile (MMA N)
constexpr int kKs = 32;       // K per MMA (bytes of int8)
constexpr int kThr = 256;     // threads per CTA
constexpr int kTmemCols = 512;
constexpr int kATile = kM * kKs;           // bytes of one digit plane of one K step (4 KB)
constexpr int kBTile = kN * kKs;           // bytes of one matrix digit plane of one K step (3 KB)
constexpr int kBStep = kS * kBTile;        // matrix digits of one (tile, K step) (15 KB)
constexpr unsigned long long kWaitCycles = 4000000000ull;  // ~2 s at 1.9 GHz

// ---- PTX helpers -----------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// K-major canonical layout without swizzle: core matrices of 8 rows x 16 bytes,
// the two 16-byte K halves of a 32-byte K step 128 bytes apart (leading byte
// offset), 8-row groups 256 bytes apart (stride byte offset); descriptor
// version 1 (sm_100), base offset 0, layout type 0
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)(128 >> 4) << 16) | ((uint64_t)(256 >> 4) << 32) |
         (1ull << 46);
}

// instruction descriptor of kind::i8: S32 accumulator, K-major A and B,
// A / B signed (1) or unsigned (0) bytes, N = kN, M = kM
__host__ __device__ constexpr uint32_t idesc_i8(int a_signed, int b_signed) {
  return (2u << 4) | ((uint32_t)a_signed << 7) | ((uint32_t)b_signed << 10) | ((uint32_t)(kN >> 3) << 17) |
         ((uint32_t)(kM >> 4) << 24);
}

__device__ __forceinline__ void mma_i8(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void mma_commit(uint64_t* mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(mbar))
               : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t* mbar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(mbar)), "r"(count) : "memory");
}

// wait for the completion of the phase with the given parity; false on a
// timeout, or at once when another CTA has already timed out (bit 1 of *flags),
// so that a kernel whose tensor-core work never completes ends within about
// one timeout instead of one per CTA
__device__ __forceinline__ bool mbar_wait(uint64_t* mbar, uint32_t parity, const unsigned* flags) {
  const uint32_t a = smem_u32(mbar);
  const unsigned long long t0 = clock64();
  for (unsigned it = 0;; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
    if (clock64() - t0 > kWaitCycles) return false;
    if ((it & 1023u) == 1023u && (*(volatile const unsigned*)flags & 2u)) return false;
  }
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// ---- digits ----------------------------------------------------------------------------
// exponent e with max < 2^e (0 for an all-zero column)
__device__ __forceinline__ int col_exponent(double mx) {
  if (!(mx > 0.0)) return 0;
  int e;
  frexp(mx, &e);
  return e;
}

// Signed base-256 digits of |m| <= 2^38: with m' = m + 0x80808080, the low four
// bytes of m' are the four lower digits plus 128 (each digit the centred
// residue in [-128, 127]) and m' >> 32 is the top digit (|top| <= 64); as int8
// bytes the lower digits are those bytes with the top bit flipped.
// Four values -> five words (one per digit plane, byte b = value b).
__device__ __forceinline__ void digits4(long long m0, long long m1, long long m2, long long m3, uint32_t (&w)[5]) {
  const long long b = 0x80808080LL;
  const long long p0 = m0 + b, p1 = m1 + b, p2 = m2 + b, p3 = m3 + b;
  const uint32_t l0 = (uint32_t)p0 ^ 0x80808080u, l1 = (uint32_t)p1 ^ 0x80808080u;
  const uint32_t l2 = (uint32_t)p2 ^ 0x80808080u, l3 = (uint32_t)p3 ^ 0x80808080u;
  const uint32_t h0 = (uint32_t)(p0 >> 32), h1 = (uint32_t)(p1 >> 32), h2 = (uint32_t)(p2 >> 32),
                 h3 = (uint32_t)(p3 >> 32);
  // 4 x 4 byte transpose of the low words: plane 4 - i gathers byte i
  const uint32_t a = __byte_perm(l0, l1, 0x5140), c = __byte_perm(l2, l3, 0x5140);
  const uint32_t e = __byte_perm(l0, l1, 0x7362), f = __byte_perm(l2, l3, 0x7362);
  w[4] = __byte_perm(a, c, 0x5410);  // byte 0 (weight 1)
  w[3] = __byte_perm(a, c, 0x7632);  // byte 1 (256)
  w[2] = __byte_perm(e, f, 0x5410);  // byte 2 (256^2)
  w[1] = __byte_perm(e, f, 0x7632);  // byte 3 (256^3)
  w[0] = __byte_perm(__byte_perm(h0, h1, 0x0040), __byte_perm(h2, h3, 0x0040), 0x5410);  // top digit
}

// 16 values (the 16 K positions of one half of a K step) -> five 16-byte digit
// rows, stored at dst + s * plane_stride; m = rint(x sc), |m| <= 2^38
__device__ __forceinline__ void store_digits16(const double (&x)[16], double sc, unsigned char* dst,
                                               int plane_stride) {
  uint32_t w[4][5];
#pragma unroll
  for (int j = 0; j < 4; ++j)
    digits4(__double2ll_rn(x[4 * j] * sc), __double2ll_rn(x[4 * j + 1] * sc), __double2ll_rn(x[4 * j + 2] * sc),
            __double2ll_rn(x[4 * j + 3] * sc), w[j]);
#pragma unroll
  for (int s = 0; s < kS; ++s)
    *reinterpret_cast<uint4*>(dst + (size_t)s * plane_stride) = make_uint4(w[0][s], w[1][s], w[2][s], w[3][s]);
}

// byte offset of (row r, k) inside one K-step tile of the canonical layout
__device__ __forceinline__ int tile_off(int r, int khalf) { return (r >> 3) * 256 + khalf * 128 + (r & 7) * 16; }

// ---- the kernel --------------------------------------------------------------------------
struct ZsArgs {
  int K, NOUT;          // contraction length and outputs per column
  int nvar;             // variables (inverse: full variables; forward: quadratic variables)
  long long ncol;       // columns per variable (NYAA NXAA)
  const double* in;     // inverse: Y2 [var][col][K]; forward: phys [full var][col][K]
  double* out;          // inverse: phys [var][col][NOUT]; forward: Q2 [q][col][NOUT]
  const unsigned char* mat;  // matrix digits [tile][kstep][plane][kN x 32 canonical]
  QuadDesc q;           // forward: the products; both: KE / timeseries objects
  const double* wz;     // Gauss-Chebyshev weights (grid z)
  const double* wzinv;  // 1 / wz
  unsigned long long* cfl_bits;  // inverse, last stage: maxima of |u|, |v|, |w| / wz
  double* ke_partial;   // forward, first stage: [cta][3]
  double* ts_partial;   // first stage: [cta][kMaxTs] (row offset ts_row0)
  long long ts_row0;
  unsigned* flags;      // bit 1: a tensor-core wait timed out
};

template <bool FWD>
__global__ void __launch_bounds__(kThr, 1) k_zsplit(ZsArgs a) {
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ uint64_t mbar[3];
  __shared__ uint32_t tmem_base_s;
  __shared__ int ok_s;
  __shared__ int cexp[kM];
  __shared__ double red[kThr / 32][4];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int var = FWD ? blockIdx.x : blockIdx.y;
  const long long col0 = (long long)(FWD ? blockIdx.y : blockIdx.x) * kM;
  const int K = a.K, NOUT = a.NOUT, nks = K / kKs, ntiles = NOUT / kN;
  unsigned char* Adig = smem;                                   // kS planes x nks x 4 KB
  unsigned char* Bbuf = smem + (size_t)kS * nks * kATile;       // 2 x 15 KB
  const int plane = nks * kATile;                               // bytes of one digit plane

  if (tid == 0) {
    mbar_init(&mbar[0], 1);
    mbar_init(&mbar[1], 1);
    mbar_init(&mbar[2], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base_s)),
                 "r"(kTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }

  // ---- pass 1: per-column maximum (and, in the forward pass, the first
  //      stage's KE / timeseries sums of this quadratic variable) ----
  const int c = tid >> 1, half = tid & 1;  // two threads per column
  const long long col = col0 + c;
  const bool colok = col < a.ncol;
  int f1 = 0, f2 = -1;
  if (FWD) {
    f1 = a.q.v1[var];
    f2 = a.q.v2[var];
    if (f1 < 0) { f1 = f2; f2 = -1; }
  }
  const double* src1 = a.in + ((size_t)(FWD ? f1 : var) * a.ncol + (colok ? col : 0)) * K;
  const double* src2 = (FWD && f2 >= 0) ? a.in + ((size_t)f2 * a.ncol + (colok ? col : 0)) * K : nullptr;
  auto value = [&](int k) -> double {
    const double x = src1[k];
    return src2 ? x * src2[k] : x;
  };
  double mx = 0.0;
  // first-stage objects on this quadratic variable: KE (uu, vv, ww) and timeseries
  double ke = 0.0, tsv[kMaxTs];
  int keslot = -1;
  if (FWD && a.ke_partial)
    for (int j = 0; j < 3; ++j)
      if (a.q.ke_q[j] == var) keslot = j;
  const bool want_ts = FWD && a.ts_partial != nullptr;
#pragma unroll
  for (int o = 0; o < kMaxTs; ++o) tsv[o] = 0.0;
  if (colok) {
    for (int k = half; k < K; k += 2) {
      const double v = value(k);
      mx = fmax(mx, fabs(v));
      if (FWD) {
        if (keslot >= 0) ke += a.wz[k] * v;
        if (want_ts) {
#pragma unroll
          for (int o = 0; o < kMaxTs; ++o)
            if (o < a.q.ts_n && a.q.ts_src[o] == -1 - var) {
              const int zs = a.q.ts_z[o];
              tsv[o] += (zs < 0) ? a.wz[k] * v : (k == zs ? v : 0.0);
            }
        }
      }
    }
  }
  mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, 1));
  if (half == 0) cexp[c] = col_exponent(mx);
  __syncthreads();
  const double sc = colok ? ldexp(1.0, 38 - cexp[c]) : 0.0;

  // ---- pass 2: digits of the whole column range into shared memory ----
  for (int ks = 0; ks < nks; ++ks) {
    double x[16];
    const int k0 = ks * kKs + half * 16;
#pragma unroll
    for (int i = 0; i < 16; ++i) x[i] = colok ? value(k0 + i) : 0.0;
    store_digits16(x, sc, Adig + (size_t)ks * kATile + tile_off(c, half), plane);
  }
  fence_proxy_async();  // generic-proxy stores -> visible to the tensor cores
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem = tmem_base_s;

  // ---- tiles of kN outputs ----
  bool ok = true;
  uint32_t use[2] = {0, 0};  // completed phases of mbar[0..1]
  uint32_t tile_phase = 0;
  // per-column diagnostics of the inverse pass
  double cmax = 0.0;
  double tinv[kMaxTs];
#pragma unroll
  for (int o = 0; o < kMaxTs; ++o) tinv[o] = 0.0;
  const int quarter = warp & 3, chalf = warp >> 2;  // TMEM lane quarter, output-column half
  const int ec = quarter * 32 + lane;               // this thread's column in the epilogue
  const long long ecol = col0 + ec;
  const int eexp = cexp[ec];
  int step = 0;
  // one thread waits on each mbarrier and shares the outcome, so that every
  // thread takes the same path (and the same barriers) after a timeout
  auto wait_shared = [&](uint64_t* mb, uint32_t parity) -> bool {
    if (tid == 0) ok_s = mbar_wait(mb, parity, a.flags) ? 1 : 0;
    __syncthreads();
    return ok_s != 0;
  };
  if (tid == 0) ok_s = (*(volatile const unsigned*)a.flags & 2u) ? 0 : 1;
  __syncthreads();
  ok = ok_s != 0;  // a CTA that starts after a timeout elsewhere does no tensor-core work
  for (int t = 0; t < ntiles && ok; ++t) {
    for (int ks = 0; ks < nks; ++ks, ++step) {
      const int b = step & 1;
      if (step >= 2) {  // the MMAs that read buffer b two steps ago are done
        if (!wait_shared(&mbar[b], use[b] & 1)) { ok = false; break; }
        ++use[b];
      }
      // matrix digits of (tile t, step ks): a straight copy of 15 KB
      const uint4* g = reinterpret_cast<const uint4*>(a.mat + ((size_t)t * nks + ks) * kBStep);
      uint4* d = reinterpret_cast<uint4*>(Bbuf + (size_t)b * kBStep);
      for (int i = tid; i < kBStep / 16; i += kThr) d[i] = __ldg(g + i);
      fence_proxy_async();
      fence_before();
      __syncthreads();
      fence_after();
      if (tid == 0) {
        const uint32_t abase = smem_u32(Adig + (size_t)ks * kATile);
        const uint32_t bbase = smem_u32(Bbuf + (size_t)b * kBStep);
#pragma unroll
        for (int i = 0; i < kS; ++i)
#pragma unroll
          for (int j = 0; j < kS - i; ++j) {
            const int dd = i + j;
            // the first product of anti-diagonal dd in this tile overwrites
            const uint32_t acc = (ks > 0 || i > 0) ? 1u : 0u;
            mma_i8(tmem + (uint32_t)(dd * kN), smem_desc(abase + (uint32_t)(i * plane)),
                   smem_desc(bbase + (uint32_t)(j * kBTile)), idesc_i8(1, 1), acc);
          }
        mma_commit(&mbar[b]);
      }
    }
    if (!ok) break;
    // all MMAs of the tile: one more commit on mbar[2] after the last step's
    if (tid == 0) mma_commit(&mbar[2]);
    if (!wait_shared(&mbar[2], tile_phase & 1)) { ok = false; break; }
    ++tile_phase;
    fence_after();
    // ---- epilogue: thread = column ec, output columns [chalf*48, chalf*48+48) of the tile ----
    const double osc = ldexp(1.0, eexp - 42);
    const bool wr = ecol < a.ncol;
    double* dst = a.out + ((size_t)var * a.ncol + (wr ? ecol : 0)) * NOUT + (size_t)t * kN;
#pragma unroll 1
    for (int j0 = chalf * (kN / 2); j0 < (chalf + 1) * (kN / 2); j0 += 16) {
      uint32_t r[kS][16];
      const uint32_t ta = tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)j0;
#pragma unroll
      for (int dd = 0; dd < kS; ++dd) tmem_ld16(ta + (uint32_t)(dd * kN), r[dd]);
      tmem_wait_ld();
      double v[16];
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        const long long S = (long long)(int)r[0][i] * 4294967296LL + (long long)(int)r[1][i] * 16777216LL +
                            (long long)(int)r[2][i] * 65536LL + (long long)(int)r[3][i] * 256LL +
                            (long long)(int)r[4][i];
        v[i] = (double)S * osc;
      }
      if (wr) {
#pragma unroll
        for (int i = 0; i < 16; i += 2) *reinterpret_cast<double2*>(dst + j0 + i) = make_double2(v[i], v[i + 1]);
        if (!FWD) {
          const int z0 = t * kN + j0;
          if (a.cfl_bits && var < 3) {
#pragma unroll
            for (int i = 0; i < 16; ++i) cmax = fmax(cmax, fabs(v[i]) * (var == 2 ? a.wzinv[z0 + i] : 1.0));
          }
          if (a.ts_partial) {
#pragma unroll
            for (int o = 0; o < kMaxTs; ++o)
              if (o < a.q.ts_n && a.q.ts_src[o] == var) {
                const int zs = a.q.ts_z[o];
                for (int i = 0; i < 16; ++i) tinv[o] += (zs < 0) ? a.wz[z0 + i] * v[i] : (z0 + i == zs ? v[i] : 0.0);
              }
          }
        }
      }
    }
    fence_before();
    __syncthreads();  // accumulators read: the next tile may overwrite them
    fence_after();
  }

  // ---- diagnostics: block totals ----
  const size_t cta = (size_t)blockIdx.y * gridDim.x + blockIdx.x;
  auto block_sum = [&](double v, bool is_max) -> double {
    for (int o = 16; o > 0; o >>= 1) {
      const double w = __shfl_xor_sync(0xffffffffu, v, o);
      v = is_max ? fmax(v, w) : v + w;
    }
    __syncthreads();
    if (lane == 0) red[warp][0] = v;
    __syncthreads();
    double s = is_max ? 0.0 : 0.0;
    for (int w = 0; w < kThr / 32; ++w) s = is_max ? fmax(s, red[w][0]) : s + red[w][0];
    return s;
  };
  if (!FWD && a.cfl_bits && var < 3) {
    const double m = block_sum(cmax, true);
    if (tid == 0) atomicMax(a.cfl_bits + var, (unsigned long long)__double_as_longlong(m));
  }
  if (a.ts_partial) {
    for (int o = 0; o < kMaxTs; ++o) {
      const double s = block_sum(FWD ? tsv[o] : tinv[o], false);
      if (tid == 0) a.ts_partial[(size_t)(a.ts_row0 + cta) * kMaxTs + o] = s;
    }
  }
  if (FWD && a.ke_partial) {
    const double s = block_sum(ke, false);
    if (tid < 3) a.ke_partial[cta * 3 + tid] = (tid == keslot) ? s : 0.0;
  }
  if (!ok && tid == 0) atomicOr(a.flags, 2u);
  fence_before();
  __syncthreads();
  if (warp == 0) {
    fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols));
  }
}

}  // namespace

// ---- host side -------------------------------------------------------------------------------
// Matrix digits in the order the kernel streams them: [tile][kstep][plane][canonical
// kN x 32 tile].  B[n][k] is the contraction matrix with outputs as rows (n < NOUT)
// and the contraction index as columns (k < K).
std::vector<unsigned char> zsplit_matrix_digits(int K, int NOUT, bool fwd, int NZAA) {
  const int nks = K / kKs, ntiles = NOUT / kN;
  std::vector<unsigned char> out((size_t)ntiles * nks * kBStep, 0);
  const long double pi = 3.141592653589793238462643383279502884L;
  for (int o = 0; o < NOUT; ++o)
    for (int k = 0; k < K; ++k) {
      long double c;
      if (fwd)  // REDFT10: row n = o, column z = k
        c = 2.0L * cosl(pi * (long double)o * (2.0L * k + 1.0L) / (2.0L * NZAA));
      else  // REDFT01: row z = o, column n = k
        c = (k == 0 ? 1.0L : 2.0L) * cosl(pi * (long double)k * (2.0L * o + 1.0L) / (2.0L * NZAA));
      const long long m = llrintl(c * 68719476736.0L);  // rint(c 2^36), |m| <= 2^37
      const int t = o / kN, r = o % kN, ks = k / kKs, kk = k % kKs;
      const size_t base = ((size_t)t * nks + ks) * kBStep + (size_t)(r >> 3) * 256 + (size_t)(kk >> 4) * 128 +
                          (size_t)(r & 7) * 16 + (size_t)(kk & 15);
      // signed base-256 digits, most significant first (the kernel's digits4)
      const long long p = m + 0x80808080LL;
      out[base] = (unsigned char)((unsigned long long)(p >> 32) & 255ull);
      for (int s = 1; s < kS; ++s)
        out[base + (size_t)s * kBTile] = (unsigned char)((((unsigned long long)p >> (8 * (4 - s))) & 255ull) ^ 0x80ull);
    }
  return out;
}

size_t zsplit_smem(int K) { return (size_t)kS * (K / kKs) * kATile + 2 * (size_t)kBStep + 1024; }

// tile divisibility, and the digits of a whole column range in shared memory
bool zsplit_supported(int NZ, int NZAA) {
  return NZ % kKs == 0 && NZAA % kKs == 0 && NZ % kN == 0 && NZAA % kN == 0 &&
         zsplit_smem(NZAA) + 4096 <= 227 * 1024;
}

size_t zsplit_ctas(long long ncol, int nvar) { return (size_t)((ncol + kM - 1) / kM) * nvar; }

// inverse: Y2 (nf variables, NZ per column) -> phys (NZAA per column)
void launch_zsplit_inv(const Dims& d, int nf, const QuadDesc& q, const double* Y2, double* phys,
                       const unsigned char* mat, const double* wz, const double* wzinv, unsigned long long* cfl_bits,
                       double* ts_partial, unsigned* flags, cudaStream_t s) {
  ZsArgs a{};
  a.K = d.NZ;
  a.NOUT = d.NZA;
  a.nvar = nf;
  a.ncol = (long long)d.NYA * d.NXA;
  a.in = Y2;
  a.out = phys;
  a.mat = mat;
  a.q = q;
  a.wz = wz;
  a.wzinv = wzinv;
  a.cfl_bits = cfl_bits;
  a.ts_partial = ts_partial;
  a.ts_row0 = 0;
  a.flags = flags;
  const size_t sm = zsplit_smem(a.K);
  cudaFuncSetAttribute(k_zsplit<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  dim3 g((unsigned)((a.ncol + kM - 1) / kM), (unsigned)nf);
  k_zsplit<false><<<g, kThr, sm, s>>>(a);
}

// forward: products of the full variables' physical columns (NZAA each) -> Q2 (NZ per column)
void launch_zsplit_fwd(const Dims& d, int nf, const QuadDesc& q, const double* phys, double* Q2,
                       const unsigned char* mat, const double* wz, double* ke_partial, double* ts_partial,
                       long long ts_row0, unsigned* flags, cudaStream_t s) {
  ZsArgs a{};
  a.K = d.NZA;
  a.NOUT = d.NZ;
  a.nvar = q.nq;
  a.ncol = (long long)d.NYA * d.NXA;
  a.in = phys;
  a.out = Q2;
  a.mat = mat;
  a.q = q;
  a.wz = wz;
  a.ke_partial = ke_partial;
  a.ts_partial = ts_partial;
  a.ts_row0 = ts_row0;
  a.flags = flags;
  (void)nf;
  const size_t sm = zsplit_smem(a.K);
  cudaFuncSetAttribute(k_zsplit<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  dim3 g((unsigned)q.nq, (unsigned)((a.ncol + kM - 1) / kM));
  k_zsplit<true><<<g, kThr, sm, s>>>(a);
}

}  // namespace coral
