// Shared device helpers for the RBM-VMC kernels (sm_100a).
//
// Scalar types: every kernel is instantiated for real RBMs (T = float) and
// holomorphic complex RBMs (T = float2, interleaved re/im, the layout of
// torch.complex64).  Spin configurations are bit-packed: bit (i & 31) of word
// (i >> 5) is 1 for spin up (s = +0.5, sigma = +1).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <math.h>

#include "../../include/qes_b200.h"

#define QES_HD __host__ __device__ __forceinline__
#define QES_D __device__ __forceinline__

#define QES_CUDA_CHECK(expr)                                   \
  do {                                                         \
    cudaError_t _e = (expr);                                   \
    if (_e != cudaSuccess) { qes_set_last_error(_e, #expr); return QES_ERR_CUDA; } \
  } while (0)

// Every kernel launch is followed by QES_LAUNCH_CHECK_N(number of launches
// since the last check); the count feeds qes_launch_count().
#define QES_LAUNCH_CHECK_N(n)                                  \
  do {                                                         \
    qes_count_launches(n);                                     \
    cudaError_t _e = cudaGetLastError();                       \
    if (_e != cudaSuccess) { qes_set_last_error(_e, "kernel launch"); return QES_ERR_CUDA; } \
  } while (0)
#define QES_LAUNCH_CHECK() QES_LAUNCH_CHECK_N(1)

void qes_set_last_error(cudaError_t e, const char* what);
void qes_set_last_message(const char* msg);
void qes_count_launches(int n);

// Per-kernel-class CUDA-event timing (enabled by qes_profile_enable): a launch site
// brackets its kernel with qes_prof_begin / qes_prof_end on the launch stream.
enum { QES_PROF_OV = 0, QES_PROF_OHU = 1, QES_PROF_REDUCE = 2, QES_PROF_GRAM = 3, QES_PROF_CHOL = 4,
       QES_PROF_SV = 5, QES_PROF_CLASSES = 6 };
bool qes_prof_on();
int qes_prof_begin(int cls, cudaStream_t st);        // returns a slot or -1
void qes_prof_end(int slot, cudaStream_t st);

// Programmatic dependent launch of the per-iteration SR kernels.  A kernel launched through
// qes_launch_pdl may start (prologue, prefetch of operands older than its predecessor) while its
// predecessor in the stream drains; pdl_wait() blocks the calling thread until the predecessor
// has completed and its writes are visible.  Every kernel on such a chain calls pdl_wait() before
// it can finish, so "the predecessor has completed" carries down the chain.  Kernels launched the
// ordinary way see both calls as no-ops.  qes_set_pdl(0) turns the attribute off.
bool qes_pdl_on();
template <class... KArgs, class... Args>
inline cudaError_t qes_launch_pdl(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                                  Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = qes_pdl_on() ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, kern, args...);
}
QES_D void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
QES_D void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// Converged flag of a CG solve, read by the matvec kernels of later iterations before they wait
// on their predecessor: once set (by the x/r update of the converging iteration) it stays set
// until the next solve's setup, so a CTA that sees it may skip its work (the solution is final);
// a CTA that reads a stale zero does the work, which nothing consumes any more.  One thread
// reads it and the block follows that thread's value.
QES_D bool cg_block_done(const double* flag) {
  __shared__ int s_done;
  if (threadIdx.x == 0) s_done = (flag != nullptr && *reinterpret_cast<const volatile double*>(flag) != 0.0) ? 1 : 0;
  __syncthreads();
  return s_done != 0;
}

// ----------------------------------------------------------------------------
// scalar algebra on float / float2
// ----------------------------------------------------------------------------
QES_HD float2 c2(float r, float i) { return make_float2(r, i); }
QES_HD float2 operator+(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
QES_HD float2 operator-(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
QES_HD float2 operator*(float2 a, float2 b) { return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
QES_HD float2 operator*(float s, float2 a) { return make_float2(s * a.x, s * a.y); }
QES_HD float2 conjf2(float2 a) { return make_float2(a.x, -a.y); }
QES_HD double2 operator+(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }

template <class T> struct ScalarTraits;
template <> struct ScalarTraits<float> {
  static constexpr bool is_complex = false;
  QES_HD static float one() { return 1.f; }
  QES_HD static float zero() { return 0.f; }
};
template <> struct ScalarTraits<float2> {
  static constexpr bool is_complex = true;
  QES_HD static float2 one() { return make_float2(1.f, 0.f); }
  QES_HD static float2 zero() { return make_float2(0.f, 0.f); }
};

QES_D float to_re(float a) { return a; }
QES_D float to_re(float2 a) { return a.x; }
QES_D float2 to_c(float a) { return make_float2(a, 0.f); }
QES_D float2 to_c(float2 a) { return a; }
QES_D float conjx(float a) { return a; }
QES_D float2 conjx(float2 a) { return conjf2(a); }
QES_D float scal(float s, float a) { return s * a; }
QES_D float2 scal(float s, float2 a) { return make_float2(s * a.x, s * a.y); }

// r = c + g * (t * s)       (one hidden-unit factor of a psi ratio)
QES_D float ratio_factor(float c, float g, float t, float s) { return fmaf(g * t, s, c); }
QES_D float2 ratio_factor(float2 c, float g, float2 t, float2 s) {
  const float tr = g * t.x, ti = g * t.y;
  float2 r;
  r.x = fmaf(tr, s.x, fmaf(-ti, s.y, c.x));
  r.y = fmaf(tr, s.y, fmaf(ti, s.x, c.y));
  return r;
}

QES_D float mulx(float a, float b) { return a * b; }
QES_D float2 mulx(float2 a, float2 b) { return a * b; }
QES_D float addx(float a, float b) { return a + b; }
QES_D float2 addx(float2 a, float2 b) { return a + b; }

// Power-of-two renormalisation of a running product: keeps |acc| in [1,2)
// and moves the binary exponent into an integer so that a product over
// thousands of hidden units can neither overflow nor underflow.
QES_D void renorm(float& acc, int& ex) {
  const float m = fabsf(acc);
  if (m > 0.f && isfinite(m)) {
    const int e = ((__float_as_int(m) >> 23) & 0xff) - 127;
    acc *= __int_as_float((127 - e) << 23);
    ex += e;
  }
}
QES_D void renorm(float2& acc, int& ex) {
  const float m = fmaxf(fabsf(acc.x), fabsf(acc.y));
  if (m > 0.f && isfinite(m)) {
    const int e = ((__float_as_int(m) >> 23) & 0xff) - 127;
    const float sc = __int_as_float((127 - e) << 23);
    acc.x *= sc; acc.y *= sc;
    ex += e;
  }
}

// exp of a (possibly complex) exponent
QES_D float expx(float z) { return expf(z); }
QES_D float2 expx(float2 z) {
  const float m = expf(z.x);
  float s, c;
  sincosf(z.y, &s, &c);
  return make_float2(m * c, m * s);
}

// log cosh on the branch  s*z + log1p(exp(-2 s z)) - log 2,  s = sign(Re z)
QES_D float log_cosh(float x) {
  const float ax = fabsf(x);
  return ax + log1pf(expf(-2.f * ax)) - 0.69314718055994531f;
}
QES_D float2 log_cosh(float2 z) {
  const float sg = (z.x < 0.f) ? -1.f : 1.f;
  const float x = sg * z.x, y = sg * z.y;          // Re >= 0
  const float em = expm1f(-2.f * x);               // q - 1,  q = exp(-2x) <= 1
  const float q = 1.f + em;
  float sy, cy;
  sincosf(y, &sy, &cy);
  // 1 + w with w = q exp(-2iy), written without cancellation near cosh(z) = 0:
  //   Re(1+w) = (1 - q) + 2 q cos^2 y,  Im(1+w) = -2 q sin y cos y
  const float r1 = -em + 2.f * q * cy * cy;
  const float i1 = -2.f * q * sy * cy;
  float re;
  if (q < 0.25f) re = 0.5f * log1pf(q * (2.f * (2.f * cy * cy - 1.f) + q));   // log|1+w|, small w
  else re = 0.5f * logf(r1 * r1 + i1 * i1);
  const float im = atan2f(i1, r1);
  return make_float2(x + re - 0.69314718055994531f, y + im);
}

// tanh, stable for large |Re z|
QES_D float tanhx(float x) { return tanhf(x); }
QES_D float2 tanhx(float2 z) {
  // tanh(x+iy) = [sign(x)(1 - q^2) + i 4 q sin y cos y] / [(1 - q)^2 + 4 q cos^2 y],
  // q = exp(-2|x|); both forms avoid cancellation near the poles (x = 0, cos y = 0)
  const float em = expm1f(-2.f * fabsf(z.x));      // q - 1
  const float q = 1.f + em;
  float sy, cy;
  sincosf(z.y, &sy, &cy);
  const float den = em * em + 4.f * q * cy * cy;
  const float re = copysignf(-em * (2.f + em), z.x) / den;
  const float im = 4.f * q * sy * cy / den;
  return make_float2(re, im);
}

// ----------------------------------------------------------------------------
// bit-packed configurations
// ----------------------------------------------------------------------------
QES_HD int n_words(int ns) { return (ns + 31) >> 5; }
QES_D float sigma_of(const uint32_t* w, int i) { return ((w[i >> 5] >> (i & 31)) & 1u) ? 1.f : -1.f; }
QES_D uint32_t bit_of(const uint32_t* w, int i) { return (w[i >> 5] >> (i & 31)) & 1u; }

// ----------------------------------------------------------------------------
// Philox4x32-10 (Salmon et al., SC'11) -- counter-based, one call per proposal
// ----------------------------------------------------------------------------
struct Philox4 { uint32_t x, y, z, w; };

QES_HD Philox4 philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0, uint32_t k1) {
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u, W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    if (r > 0) { k0 += W0; k1 += W1; }
    const uint64_t p0 = (uint64_t)M0 * c0;
    const uint64_t p1 = (uint64_t)M1 * c2;
    const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    const uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
    c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
  }
  Philox4 o; o.x = c0; o.y = c1; o.z = c2; o.w = c3;
  return o;
}

QES_HD uint32_t bounded_u32(uint32_t r, uint32_t n) { return (uint32_t)(((uint64_t)r * n) >> 32); }
// (0,1) uniform, exactly representable in float32
QES_HD float uniform_open(uint32_t r) { return ((float)(r >> 9) + 0.5f) * 1.1920928955078125e-07f; }

enum { QES_STREAM_PROPOSAL = 0, QES_STREAM_INIT_RND = 1, QES_STREAM_INIT_FIXED = 2 };

// ----------------------------------------------------------------------------
// warp helpers
// ----------------------------------------------------------------------------
QES_D float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
QES_D float2 warp_sum(float2 v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
    v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
  }
  return v;
}
QES_D double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
