// Stochastic reconfiguration with the RBM's structured log-derivatives.
//
// For the RBM, O_s = [sigma_s, t_s, sigma_s (x) t_s] with t = tanh(theta), so
//   (O v)_s    = sigma_s . v_a + t_s . (v_b + V^T sigma_s)        (V = v_W, ns x nh)
//   (O^H u)_W  = Sigma^T diag(u) conj(T),  (O^H u)_a = Sigma^T u,  (O^H u)_b = T^H u
// and the SR matrix is applied as S v = O_c^H O_c v / Ns = O^H (w - mean w) / Ns
// with w = O v (the centred u sums to zero, so O^H u = O_c^H u).  O (Ns x P)
// is never formed: one matvec reads the packed spins and T (Ns x nh) only.
//
// Precision: per-chunk sums in float32, chunk partials and every CG vector,
// dot product and scalar in float64 (the reference promotes SR data to
// float64, tdvp.py:827-858).  CG follows SciPy's rule ||r|| <= max(rtol*||b||,
// atol); the device freezes x at the first iteration that meets it, so the
// result does not depend on how often the host checks.
#include "common.cuh"
#include "sr_tc.h"

#include <algorithm>
#include <atomic>
#include <vector>

// 0 = tensor cores when the shapes allow it, 1 = CUDA cores only (float32), 2 = tensor cores required,
// 3 = CUDA cores with float64 contractions (the reference's SR precision, for accuracy checks)
static std::atomic<int> g_sr_impl{0};
extern "C" int qes_set_sr_impl(int impl) {
  if (impl < 0 || impl > 3) {
    qes_set_last_message("qes_set_sr_impl: impl must be 0 (auto), 1 (cuda cores), 2 (tensor cores) or 3 (float64)");
    return QES_ERR_ARG;
  }
  g_sr_impl.store(impl);
  return QES_OK;
}

#define QES_ARG_CHECK(cond, msg) do { if (!(cond)) { qes_set_last_message(msg); return QES_ERR_ARG; } } while (0)

// SM count of the current device (cached per device)
static int qes_sm_count() {
  static int cache[64] = {0};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
  if (cache[dev] == 0) {
    int n = 0;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
    cache[dev] = n;
  }
  return cache[dev];
}

template <class T> struct VecT;
template <> struct VecT<float> { using type = double; };
template <> struct VecT<float2> { using type = double2; };

QES_HD double vzero(double) { return 0.0; }
QES_HD double2 vzero(double2) { return make_double2(0.0, 0.0); }
QES_D float to_f(double v) { return (float)v; }
QES_D float2 to_f(double2 v) { return make_float2((float)v.x, (float)v.y); }
QES_D double to_d(float v) { return (double)v; }
QES_D double2 to_d(float2 v) { return make_double2(v.x, v.y); }
QES_D double to_d(double v) { return v; }
QES_D double2 to_d(double2 v) { return v; }
template <class T> struct IsF64 { static constexpr bool value = false; };
template <> struct IsF64<double> { static constexpr bool value = true; };
template <> struct IsF64<double2> { static constexpr bool value = true; };
QES_D double vadd(double a, double b) { return a + b; }
QES_D double2 vadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
QES_D double vscale(double s, double a) { return s * a; }
QES_D double2 vscale(double s, double2 a) { return make_double2(s * a.x, s * a.y); }
QES_D double2 vscale(double2 s, double2 a) { return make_double2(s.x * a.x - s.y * a.y, s.x * a.y + s.y * a.x); }
QES_D double vdotc(double a, double b) { return a * b; }                       // conj(a) b, real part only
QES_D double vdotc(double2 a, double2 b) { return a.x * b.x + a.y * b.y; }     // Re(conj(a) b)
// element from the complex eloc / w buffer in the working scalar type
QES_D float from_c(float2 v, float) { return v.x; }
QES_D float2 from_c(float2 v, float2) { return v; }

// ----------------------------------------------------------------------------
// mean of a complex float32 vector in float64 -> out[0..1]  (one block)
// ----------------------------------------------------------------------------
constexpr int MEAN_THREADS = 1024;
__global__ void __launch_bounds__(MEAN_THREADS) mean_c_kernel(int64_t n, const float2* __restrict__ w,
                                                              double* __restrict__ out,
                                                              const float* __restrict__ wts = nullptr) {
  double sr = 0, si = 0;
  for (int64_t k = threadIdx.x; k < n; k += blockDim.x) {
    const double f = wts ? (double)wts[k] : 1.0;           // sum wts w / Ns: the weighted mean
    sr += f * w[k].x;
    si += f * w[k].y;
  }
  __shared__ double rr[MEAN_THREADS / 32], ri[MEAN_THREADS / 32];
  sr = warp_sum(sr); si = warp_sum(si);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) { rr[warp] = sr; ri[warp] = si; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0, b = 0;
    for (int q = 0; q < MEAN_THREADS / 32; ++q) { a += rr[q]; b += ri[q]; }
    out[0] = a / (double)n;
    out[1] = b / (double)n;
  }
}

// ----------------------------------------------------------------------------
// CUDA-core forms: register-tiled contractions.  The spins are staged in shared memory as +-1
// reals, so every sign x value product is one FMA.  Block 32 x 8 threads; a thread owns R rows x
// PT_C columns of the output tile, columns interleaved by 32 (conflict-free shared-memory loads),
// rows interleaved by 8 (all lanes of a warp read the same spin: a broadcast).  The accumulator
// type A is float / float2 in the plain-FP32 form and double / double2 in the float64 form (the
// same float32 T promoted, the reference's SR precision); K is the contraction slice per pass.
// ----------------------------------------------------------------------------
constexpr int PT_TX = 32, PT_TY = 8, PT_C = 4;
constexpr int PT_THREADS = PT_TX * PT_TY;
constexpr int PT_U = PT_TX * PT_C;            // columns (hidden units) per block
constexpr int PT_K = 32;                      // contraction slice staged per pass (float32 accumulators)
constexpr int PT_K64 = 16;                    // ... (float64 accumulators)
constexpr int PT_SPLIT = 512;                 // samples per O^H u split (one partial P-vector each)

// accumulator traits: RA = real type, W = complex type of the per-sample vectors w / u
template <class A> struct Acc;
template <> struct Acc<float> { using RA = float; using W = float2; };
template <> struct Acc<float2> { using RA = float; using W = float2; };
template <> struct Acc<double> { using RA = double; using W = double2; };
template <> struct Acc<double2> { using RA = double; using W = double2; };

QES_D float acc_cv(float x, float) { return x; }
QES_D float acc_cv(double x, float) { return (float)x; }
QES_D float2 acc_cv(float2 x, float2) { return x; }
QES_D float2 acc_cv(double2 x, float2) { return make_float2((float)x.x, (float)x.y); }
QES_D double acc_cv(float x, double) { return (double)x; }
QES_D double acc_cv(double x, double) { return x; }
QES_D double2 acc_cv(float2 x, double2) { return make_double2(x.x, x.y); }
QES_D double2 acc_cv(double2 x, double2) { return x; }
QES_D float2 acc_to_w(float x) { return make_float2(x, 0.f); }
QES_D float2 acc_to_w(float2 x) { return x; }
QES_D double2 acc_to_w(double x) { return make_double2(x, 0.0); }
QES_D double2 acc_to_w(double2 x) { return x; }
QES_D float acc_from_w(float2 w, float) { return w.x; }
QES_D float2 acc_from_w(float2 w, float2) { return w; }
QES_D double acc_from_w(float2 w, double) { return (double)w.x; }
QES_D double2 acc_from_w(float2 w, double2) { return make_double2(w.x, w.y); }
QES_D double acc_from_w(double2 w, double) { return w.x; }
QES_D double2 acc_from_w(double2 w, double2) { return w; }
QES_D float fma_s(float s, float v, float a) { return fmaf(s, v, a); }
QES_D float2 fma_s(float s, float2 v, float2 a) { return make_float2(fmaf(s, v.x, a.x), fmaf(s, v.y, a.y)); }
QES_D double fma_s(double s, double v, double a) { return fma(s, v, a); }
QES_D double2 fma_s(double s, double2 v, double2 a) { return make_double2(fma(s, v.x, a.x), fma(s, v.y, a.y)); }
QES_D float amul(float a, float b) { return a * b; }
QES_D float2 amul(float2 a, float2 b) { return a * b; }
QES_D double amul(double a, double b) { return a * b; }
QES_D double2 amul(double2 a, double2 b) { return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
QES_D float aadd(float a, float b) { return a + b; }
QES_D float2 aadd(float2 a, float2 b) { return a + b; }
QES_D double aadd(double a, double b) { return a + b; }
QES_D double2 aadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
QES_D float aconj(float a) { return a; }
QES_D float2 aconj(float2 a) { return conjf2(a); }
QES_D double aconj(double a) { return a; }
QES_D double2 aconj(double2 a) { return make_double2(a.x, -a.y); }
template <class A> QES_D A azero() { return acc_cv(0.f, A()); }
template <> QES_D float2 azero<float2>() { return make_float2(0.f, 0.f); }
template <> QES_D double2 azero<double2>() { return make_double2(0.0, 0.0); }
QES_D double2 warp_sum(double2 v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
    v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
  }
  return v;
}

// wpart[ub][s] = sum over the hidden units j of block ub of t_sj (v_b,j + sum_i sigma_si V_ij),
// plus sigma_s . v_a in unit block 0: z = Sigma V is accumulated in registers over K-site slices
// (spins from one word per sample and slice), then folded with t and summed over the warp's lanes.
template <class T, class A, class V, int R, int K>
__global__ void __launch_bounds__(PT_THREADS) ov_tile_kernel(int ns, int nh, int64_t n_samples,
                                                             const uint32_t* __restrict__ bits,
                                                             const T* __restrict__ tanh_theta,
                                                             const V* __restrict__ v,
                                                             typename Acc<A>::W* __restrict__ wpart,
                                                             const double* __restrict__ cg_done) {
  using RA = typename Acc<A>::RA;
  constexpr int S = PT_TY * R;                   // samples per block
  __shared__ RA sg[K][S];
  __shared__ A vs[K][PT_U];
  if (cg_done && *cg_done != 0.0) return;        // converged CG (stream order: exact)
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * PT_TX + tx;
  const int64_t s0 = (int64_t)blockIdx.x * S;
  const int j0 = blockIdx.y * PT_U;
  const int nw = n_words(ns);
  const V* va = v;
  const V* vb = v + ns;
  const V* vW = v + ns + nh;
  A z[R][PT_C];
#pragma unroll
  for (int r = 0; r < R; ++r)
#pragma unroll
    for (int c = 0; c < PT_C; ++c) z[r][c] = azero<A>();
  for (int i0 = 0; i0 < ns; i0 += K) {           // K divides 32: a slice lies in one spin word
    __syncthreads();                             // the previous slice is consumed
    for (int e = tid; e < K * S; e += PT_THREADS) {
      const int sl = e % S, il = e / S;
      const int64_t s = s0 + sl;
      const int i = i0 + il;
      RA x = (RA)0;
      if (s < n_samples && i < ns) x = ((__ldg(bits + s * nw + (i >> 5)) >> (i & 31)) & 1u) ? (RA)1 : (RA)-1;
      sg[il][sl] = x;
    }
    for (int e = tid; e < K * PT_U; e += PT_THREADS) {
      const int il = e / PT_U, jl = e % PT_U;
      const int i = i0 + il, j = j0 + jl;
      vs[il][jl] = (i < ns && j < nh) ? acc_cv(vW[(int64_t)i * nh + j], A()) : azero<A>();
    }
    __syncthreads();
#pragma unroll 8
    for (int il = 0; il < K; ++il) {
      RA sv[R];
      A q[PT_C];
#pragma unroll
      for (int r = 0; r < R; ++r) sv[r] = sg[il][r * PT_TY + ty];
#pragma unroll
      for (int c = 0; c < PT_C; ++c) q[c] = vs[il][c * PT_TX + tx];
#pragma unroll
      for (int r = 0; r < R; ++r)
#pragma unroll
        for (int c = 0; c < PT_C; ++c) z[r][c] = fma_s(sv[r], q[c], z[r][c]);
    }
  }
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int64_t s = s0 + r * PT_TY + ty;
    A acc = azero<A>();
    if (s < n_samples) {
#pragma unroll
      for (int c = 0; c < PT_C; ++c) {
        const int j = j0 + c * PT_TX + tx;
        if (j < nh)
          acc = aadd(acc, amul(acc_cv(tanh_theta[s * nh + j], A()), aadd(z[r][c], acc_cv(vb[j], A()))));
      }
      if (blockIdx.y == 0) {                     // sigma_s . v_a, lanes over the sites
        for (int i = tx; i < ns; i += PT_TX) {
          const bool up = (__ldg(bits + s * nw + (i >> 5)) >> (i & 31)) & 1u;
          acc = fma_s(up ? (RA)1 : (RA)-1, acc_cv(va[i], A()), acc);
        }
      }
    }
    acc = warp_sum(acc);
    if (tx == 0 && s < n_samples) wpart[(int64_t)blockIdx.y * n_samples + s] = acc_to_w(acc);
  }
}

// w = sum of the unit-block partials (fixed order); mean of w in float64 (weighted by wts, which sum
// to Ns, when given) when wmean is given
template <class W>
__global__ void __launch_bounds__(1024) wsum_kernel(int64_t n, int nub, const W* __restrict__ wpart,
                                                     W* __restrict__ w, double* __restrict__ wmean,
                                                     const double* __restrict__ cg_done,
                                                     const float* __restrict__ wts) {
  if (cg_done && *cg_done != 0.0) return;
  double sr = 0, si = 0;
  for (int64_t k = threadIdx.x; k < n; k += blockDim.x) {
    W a = wpart[k];
    for (int b = 1; b < nub; ++b) a = aadd(a, wpart[(int64_t)b * n + k]);
    w[k] = a;
    const double f = wts ? (double)wts[k] : 1.0;
    sr += f * a.x;
    si += f * a.y;
  }
  if (!wmean) return;
  __shared__ double rr[32], ri[32];
  sr = warp_sum(sr);
  si = warp_sum(si);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) { rr[warp] = sr; ri[warp] = si; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0, b = 0;
    for (int q = 0; q < (int)(blockDim.x >> 5); ++q) { a += rr[q]; b += ri[q]; }
    wmean[0] = a / (double)n;
    wmean[1] = b / (double)n;
  }
}

// partial[split] = Sigma~^T Q~ over PT_SPLIT samples: rows are the sites plus a ones row at site
// ns (-> g_b), columns the hidden units plus a virtual unit at nh carrying u itself (-> g_a);
// Q_sj = conj(t_sj) u_s with u_s = wts_s (w_s - mean) * scale (wts_s = 1 without weights), staged
// K samples at a time.  WI: the type of the per-sample input w (complex64 E_loc or O v of the form).
template <class T, class A, class WI, int R, int K>
__global__ void __launch_bounds__(PT_THREADS) ohu_tile_kernel(int ns, int nh, int64_t n_samples,
                                                              const uint32_t* __restrict__ bits,
                                                              const T* __restrict__ tanh_theta,
                                                              const WI* __restrict__ w,
                                                              const double* __restrict__ wmean, double scale,
                                                              A* __restrict__ partial,
                                                              const double* __restrict__ cg_done,
                                                              const float* __restrict__ wts) {
  using RA = typename Acc<A>::RA;
  constexpr int IB = PT_TY * R;                  // sites per block
  __shared__ RA sg[K][IB];
  __shared__ A qs[K][PT_U];
  __shared__ A us[K];
  if (cg_done && *cg_done != 0.0) return;
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * PT_TX + tx;
  const int j0 = blockIdx.x * PT_U, i0 = blockIdx.y * IB;
  const int64_t sbeg = (int64_t)blockIdx.z * PT_SPLIT;
  const int64_t send = min(n_samples, sbeg + PT_SPLIT);
  const int nw = n_words(ns);
  const double mr = wmean ? wmean[0] : 0.0, mi = wmean ? wmean[1] : 0.0;
  A acc[R][PT_C];
#pragma unroll
  for (int r = 0; r < R; ++r)
#pragma unroll
    for (int c = 0; c < PT_C; ++c) acc[r][c] = azero<A>();
  for (int64_t c0 = sbeg; c0 < send; c0 += K) {
    const int nc = (int)min((int64_t)K, send - c0);
    __syncthreads();                             // the previous sub-chunk is consumed
    if (tid < K) {
      A u = azero<A>();
      if (tid < nc) {
        const WI wv = w[c0 + tid];
        const double f = wts ? scale * (double)wts[c0 + tid] : scale;
        // float32 forms: (w - mean) * scale in float32, as before; float64 form: all in float64
        if constexpr (sizeof(RA) == 4)
          u = acc_from_w(make_float2(((float)wv.x - (float)mr) * (float)f, ((float)wv.y - (float)mi) * (float)f), A());
        else
          u = acc_from_w(make_double2(((double)wv.x - mr) * f, ((double)wv.y - mi) * f), A());
      }
      us[tid] = u;
    }
    for (int e = tid; e < K * IB; e += PT_THREADS) {
      const int sl = e / IB, il = e % IB, i = i0 + il;
      RA x = (RA)0;
      if (sl < nc) {
        if (i < ns) x = ((__ldg(bits + (c0 + sl) * nw + (i >> 5)) >> (i & 31)) & 1u) ? (RA)1 : (RA)-1;
        else if (i == ns) x = (RA)1;
      }
      sg[sl][il] = x;
    }
    __syncthreads();                             // us
    for (int e = tid; e < K * PT_U; e += PT_THREADS) {
      const int sl = e / PT_U, jl = e % PT_U, j = j0 + jl;
      A q = azero<A>();
      if (sl < nc) {
        if (j < nh) q = amul(aconj(acc_cv(tanh_theta[(c0 + sl) * nh + j], A())), us[sl]);
        else if (j == nh) q = us[sl];
      }
      qs[sl][jl] = q;
    }
    __syncthreads();
#pragma unroll 8
    for (int sl = 0; sl < K; ++sl) {
      RA sv[R];
      A q[PT_C];
#pragma unroll
      for (int r = 0; r < R; ++r) sv[r] = sg[sl][r * PT_TY + ty];
#pragma unroll
      for (int c = 0; c < PT_C; ++c) q[c] = qs[sl][c * PT_TX + tx];
#pragma unroll
      for (int r = 0; r < R; ++r)
#pragma unroll
        for (int c = 0; c < PT_C; ++c) acc[r][c] = fma_s(sv[r], q[c], acc[r][c]);
    }
  }
  const int64_t P = (int64_t)ns + nh + (int64_t)ns * nh;
  A* out = partial + (int64_t)blockIdx.z * P;
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int i = i0 + r * PT_TY + ty;
#pragma unroll
    for (int c = 0; c < PT_C; ++c) {
      const int j = j0 + c * PT_TX + tx;
      if (i < ns && j < nh) out[ns + nh + (int64_t)i * nh + j] = acc[r][c];
      else if (i == ns && j < nh) out[ns + j] = acc[r][c];
      else if (i < ns && j == nh) out[i] = acc[r][c];
    }
  }
}

// row-tile heights: 8 rows per thread where the sites or samples are many (fewer re-reads of
// the column operand), 4 otherwise
static int pt_rows_ov(int64_t n_samples) { return n_samples >= 64 * 148 ? 8 : 4; }
static int pt_rows_ohu(int ns) { return ns + 1 > 64 ? 8 : 4; }

constexpr int OHU_SPLIT_SAMPLES = 256;           // samples per split of the batched O^H u

// sum the split partials in float64; optional  y = G + shift * p  and  dot partials of p^H y.
// A block covers cv column vectors (16 bytes: 2 complex / 4 real columns when VEC, else one
// column) x RS_THREADS / cv split groups; each thread issues the loads of up to RS_BATCH splits
// before it sums any of them, so that a block needs one round trip to L2 when
// nsplit <= groups * RS_BATCH.  The host picks cv so that the grid is about two resident blocks
// per SM.  Sums run in a fixed order (deterministic).
constexpr int RED_THREADS = 256;
constexpr int RED_BLOCKS = 296;          // grid of the element-wise CG kernels
constexpr int RS_THREADS = 512, RS_BATCH = 12;
constexpr int RS_MAX_BLOCKS = 1184;      // upper bound of dot partials written by the reduction

QES_D void acc4(double* g, float4 q) { g[0] += q.x; g[1] += q.y; g[2] += q.z; g[3] += q.w; }
QES_D void acc4(double2* g, float4 q) { g[0].x += q.x; g[0].y += q.y; g[1].x += q.z; g[1].y += q.w; }

// Dot partials of a split-reduction block and, in the last block to finish, the CG scalars:
// alpha (standard steps) or the Chronopoulos-Gear step's scalars (cgmode).
template <bool CG>
QES_D void reduce_splits_tail(const double (&dd)[5], double* __restrict__ dot_part,
                              double* __restrict__ scal, unsigned int* __restrict__ counter) {
  if (!dot_part) return;
  const int tid = threadIdx.x;
  // dot partials: dd[q] of block b at dot_part[q * RS_MAX_BLOCKS + b]
  constexpr bool cgmode = CG;
  constexpr int nd = CG ? 5 : 1;
  __shared__ double sred[5][RS_THREADS / 32];
  __shared__ bool last;
#pragma unroll
  for (int q = 0; q < 5; ++q) {
    if (q >= nd) break;
    const double v = warp_sum(dd[q]);
    if ((tid & 31) == 0) sred[q][tid >> 5] = v;
  }
  __syncthreads();
  if (tid == 0) {
#pragma unroll
    for (int q = 0; q < 5; ++q) {
      if (q >= nd) break;
      double s = 0.0;
      for (int w = 0; w < RS_THREADS / 32; ++w) s += sred[q][w];
      dot_part[q * RS_MAX_BLOCKS + blockIdx.x] = s;
    }
    // the last block to finish sums the dot partials: pAp and alpha = rr / pAp
    if (scal) {
      __threadfence();
      last = (atomicAdd(counter, 1u) == gridDim.x - 1);
    }
  }
  if (!scal) return;
  __syncthreads();
  if (!last) return;
  __threadfence();
#pragma unroll
  for (int q = 0; q < 5; ++q) {
    if (q >= nd) break;
    double v = 0.0;
    for (int b = tid; b < (int)gridDim.x; b += RS_THREADS) v += ((volatile double*)dot_part)[q * RS_MAX_BLOCKS + b];
    v = warp_sum(v);
    __syncthreads();
    if ((tid & 31) == 0) sred[q][tid >> 5] = v;
  }
  __syncthreads();
  if (tid == 0) {
    double tot[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    for (int q = 0; q < nd; ++q)
      for (int w = 0; w < RS_THREADS / 32; ++w) tot[q] += sred[q][w];
    if (!cgmode) {
      const double pap = tot[0];
      scal[1] = pap;
      scal[7] = (scal[4] == 0.0 && pap > 0.0) ? scal[0] / pap : 0.0;
    } else if (scal[4] == 0.0) {
      // Chronopoulos-Gear step k on r_k (v = r_k, y = A r_k): rr = |r_k|^2 from the vector itself,
      // the convergence test on it (x_k is final: this step's update is skipped), else
      // beta_k = rr / rr_{k-1} and alpha_k = rr / p_k^H A p_k with p_k^H A p_k expanded bilinearly
      // in p_k = r_k + beta p_{k-1}, s_k = A r_k + beta s_{k-1} (the update kernel's recurrences):
      // r^H A r + beta (Re r^H s_{k-1} + Re p_{k-1}^H A r) + beta^2 Re p_{k-1}^H s_{k-1}, from the
      // vectors themselves rather than from the orthogonality relations of exact arithmetic
      const double rw = tot[0], rr = tot[1];
      scal[2] = rr;
      if (rr <= scal[3]) {
        scal[4] = 1.0;
      } else {
        const bool first = scal[5] == 0.0;
        const double beta = (first || scal[0] <= 0.0) ? 0.0 : rr / scal[0];
        const double den = first ? rw : rw + beta * (tot[2] + tot[3]) + beta * beta * tot[4];
        scal[1] = den;                                   // p_k^H A p_k
        scal[7] = den > 0.0 ? rr / den : 0.0;
        scal[8] = beta;
        scal[0] = rr;
        scal[5] += 1.0;
      }
    }
    *counter = 0u;
  }
}

template <class T, class V, bool VEC, bool CG>
__global__ void __launch_bounds__(RS_THREADS, 2) reduce_splits_kernel(int64_t P, int nsplit, int cv,
                                                                      const T* __restrict__ partial, double shift,
                                                                      const V* __restrict__ p, V* __restrict__ y,
                                                                      double* __restrict__ dot_part,
                                                                      double* __restrict__ scal,
                                                                      unsigned int* __restrict__ counter,
                                                                      const double* __restrict__ cg_done,
                                                                      const V* __restrict__ pold,
                                                                      const V* __restrict__ sold) {
  constexpr int E = VEC ? (int)(16 / sizeof(T)) : 1;      // columns per vector
  __shared__ V red[RS_THREADS * E];                        // [split group][column vector][E]
  pdl_trigger();
  pdl_wait();                                              // the partials: previous kernel
  if (cg_done && *cg_done != 0.0) return;                  // converged CG: y is not read any more
  const int tid = threadIdx.x;
  const int groups = RS_THREADS / cv, c = tid % cv, sg = tid / cv;
  const int64_t nvec = P / E;                              // P % E == 0 when VEC
  // dd[0] = Re v^H y; with pold / sold (a Chronopoulos-Gear CG step: v = r_k, y = A r_k, the previous
  // direction p_{k-1} and s_{k-1} = A p_{k-1}): dd[1] = |v|^2, dd[2] = Re v^H s_{k-1},
  // dd[3] = Re p_{k-1}^H y, dd[4] = Re p_{k-1}^H s_{k-1}
  constexpr bool cgmode = CG;
  double dd[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  for (int64_t v0 = (int64_t)blockIdx.x * cv; v0 < nvec; v0 += (int64_t)gridDim.x * cv) {
    const int64_t vi = v0 + c;
    V g[E];
#pragma unroll
    for (int e = 0; e < E; ++e) g[e] = vzero(V());
    if (sg < groups && vi < nvec) {
      for (int z0 = sg; z0 < nsplit; z0 += groups * RS_BATCH) {
        if constexpr (VEC) {
          float4 q[RS_BATCH];
          const float4* src = reinterpret_cast<const float4*>(partial) + vi;
#pragma unroll
          for (int b = 0; b < RS_BATCH; ++b) {
            const int z = z0 + b * groups;
            q[b] = (z < nsplit) ? __ldcg(src + (int64_t)z * nvec) : make_float4(0.f, 0.f, 0.f, 0.f);
          }
#pragma unroll
          for (int b = 0; b < RS_BATCH; ++b) acc4(g, q[b]);
        } else {
          T q[RS_BATCH];
#pragma unroll
          for (int b = 0; b < RS_BATCH; ++b) {
            const int z = z0 + b * groups;
            q[b] = (z < nsplit) ? partial[(int64_t)z * P + vi] : T{};
          }
#pragma unroll
          for (int b = 0; b < RS_BATCH; ++b) g[0] = vadd(g[0], to_d(q[b]));
        }
      }
    }
    if (sg < groups) {
#pragma unroll
      for (int e = 0; e < E; ++e) red[(sg * cv + c) * E + e] = g[e];
    }
    __syncthreads();
    if (tid < cv * E) {
      const int64_t kk = v0 * E + tid;
      if (kk < P) {
        V t = red[tid];
        for (int q = 1; q < groups; ++q) t = vadd(t, red[q * cv * E + tid]);
        if (p) {
          const V pk = p[kk];
          t = vadd(t, vscale(shift, pk));
          dd[0] += vdotc(pk, t);
          if constexpr (cgmode) {
            const V po = pold[kk], so = sold[kk];
            dd[1] += vdotc(pk, pk);
            dd[2] += vdotc(pk, so);
            dd[3] += vdotc(po, t);
            dd[4] += vdotc(po, so);
          }
        }
        y[kk] = t;
      }
    }
    __syncthreads();
  }
  reduce_splits_tail<CG>(dd, dot_part, scal, counter);
}

// The same split reduction with the partials moved by bulk copies: a block's column slice of every
// split (cv 16-byte vectors each) lands in shared memory through one mbarrier, so the loads do
// not wait in the threads' scoreboards (the register-load form is bound by load latency: 24 MB of
// partials at about 2 TB/s on the 10x10 workload).  Same sums in the same fixed order as
// reduce_splits_kernel<VEC = true>, so the results are bit-identical.  A bounded wait that runs
// out records QES_ERR_TIMEOUT in *err and the block goes on with what it has.
template <class T, class V, bool CG>
__global__ void __launch_bounds__(RS_THREADS, 2) reduce_splits_bulk_kernel(int64_t P, int nsplit, int cv,
                                                                          const T* __restrict__ partial,
                                                                          double shift, const V* __restrict__ p,
                                                                          V* __restrict__ y,
                                                                          double* __restrict__ dot_part,
                                                                          double* __restrict__ scal,
                                                                          unsigned int* __restrict__ counter,
                                                                          const double* __restrict__ cg_done,
                                                                          const V* __restrict__ pold,
                                                                          const V* __restrict__ sold,
                                                                          int* __restrict__ err) {
  constexpr int E = (int)(16 / sizeof(T));
  extern __shared__ __align__(128) uint8_t rs_smem[];
  float4* sbuf = reinterpret_cast<float4*>(rs_smem);      // [split][cv]
  __shared__ V red[RS_THREADS * E];
  __shared__ __align__(8) uint64_t bar;
  pdl_trigger();
  pdl_wait();                                              // the partials: previous kernel
  if (cg_done && *cg_done != 0.0) return;
  const int tid = threadIdx.x;
  const int groups = RS_THREADS / cv, c = tid % cv, sg = tid / cv;
  const int64_t nvec = P / E;
  if (tid == 0) {
    umma::mbar_init(&bar, 1);
    umma::fence_mbar_init();
  }
  __syncthreads();
  constexpr bool cgmode = CG;
  double dd[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  uint32_t phase = 0;
  for (int64_t v0 = (int64_t)blockIdx.x * cv; v0 < nvec; v0 += (int64_t)gridDim.x * cv) {
    const int cvv = (int)((nvec - v0 < cv) ? (nvec - v0) : cv);
    if (tid == 0) {
      umma::fence_proxy_async_smem();                      // earlier reads of sbuf before the new copies
      umma::mbar_arrive_expect_tx(&bar, (uint32_t)(nsplit * cvv * 16));
      const float4* src = reinterpret_cast<const float4*>(partial) + v0;
      for (int z = 0; z < nsplit; ++z)
        umma::bulk_g2s(sbuf + (size_t)z * cv, src + (int64_t)z * nvec, (uint32_t)(cvv * 16), &bar);
    }
    if (!umma::mbar_wait(&bar, phase, 1u << 22) && tid == 0 && err) atomicCAS(err, 0, QES_ERR_TIMEOUT);
    phase ^= 1u;
    V g[E];
#pragma unroll
    for (int e = 0; e < E; ++e) g[e] = vzero(V());
    if (sg < groups && c < cvv) {
      // the same split order as the register-load form (z = sg, sg + groups, ...)
#pragma unroll 4
      for (int z = sg; z < nsplit; z += groups) acc4(g, sbuf[(size_t)z * cv + c]);
    }
    if (sg < groups) {
#pragma unroll
      for (int e = 0; e < E; ++e) red[(sg * cv + c) * E + e] = g[e];
    }
    __syncthreads();
    if (tid < cv * E) {
      const int64_t kk = v0 * E + tid;
      if (kk < P) {
        V t = red[tid];
        for (int q = 1; q < groups; ++q) t = vadd(t, red[q * cv * E + tid]);
        if (p) {
          const V pk = p[kk];
          t = vadd(t, vscale(shift, pk));
          dd[0] += vdotc(pk, t);
          if constexpr (cgmode) {
            const V po = pold[kk], so = sold[kk];
            dd[1] += vdotc(pk, pk);
            dd[2] += vdotc(pk, so);
            dd[3] += vdotc(po, t);
            dd[4] += vdotc(po, so);
          }
        }
        y[kk] = t;
      }
    }
    __syncthreads();
  }
  reduce_splits_tail<CG>(dd, dot_part, scal, counter);
}

// the bulk-copy split reduction (qes_set_reduce_bulk) where a block's slices fit 88 KB of shared
// memory (two blocks per SM): off by default -- one thread issuing a small bulk copy per split
// (147 x 560 B per block on the 10x10 workload) made the reduction slower, 16.8 against 12.8 us
// per launch (CG iteration 43.4 against 42.2 us; 6x6 J1-J2 30.2 against 28.7 us)
static std::atomic<int> g_reduce_bulk{0};
constexpr size_t kReduceBulkSmem = 88 * 1024;
extern "C" int qes_set_reduce_bulk(int on) {
  g_reduce_bulk.store(on ? 1 : 0);
  return QES_OK;
}

// y = sum of the nsplit partial P-vectors (+ shift * p, dot partials, alpha): the vector form
// when every split row starts on a 16-byte boundary
template <class T, class V>
static int launch_reduce_splits(int64_t P, int nsplit, const void* partial, double shift, const V* p, V* y,
                                double* dot_part, double* scal, unsigned int* counter, cudaStream_t st,
                                const double* cg_done = nullptr, const V* pold = nullptr,
                                const V* sold = nullptr) {
  constexpr int EV = (int)(16 / sizeof(T));
  const bool vec = !IsF64<T>::value && (P % EV == 0) && ((reinterpret_cast<uintptr_t>(partial) & 15) == 0);
  const int64_t nvec = vec ? P / EV : P;
  const int target = 2 * qes_sm_count();                   // two resident blocks per SM
  int64_t cv = (nvec + target - 1) / target;
  cv = std::max<int64_t>(cv, RS_THREADS / std::max(nsplit, 1));            // no idle split groups
  const int64_t need = (nsplit + RS_BATCH - 1) / RS_BATCH;                  // groups for one batch
  cv = std::min<int64_t>(cv, std::max<int64_t>(RS_THREADS / std::max<int64_t>(need, 1), 1));
  cv = std::max<int64_t>(1, std::min<int64_t>(cv, 128));
  const int grid = (int)std::min<int64_t>((nvec + cv - 1) / cv, RS_MAX_BLOCKS);
  const bool cg = pold != nullptr;
  if constexpr (!IsF64<T>::value) {
    const size_t bulk_smem = (size_t)nsplit * (size_t)cv * 16;
    if (vec && g_reduce_bulk.load() != 0 && bulk_smem <= kReduceBulkSmem) {
      static bool attr_set = false;                        // per process (the attribute is per function)
      if (!attr_set) {
        QES_CUDA_CHECK(cudaFuncSetAttribute(reduce_splits_bulk_kernel<T, V, false>,
                                            cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kReduceBulkSmem));
        QES_CUDA_CHECK(cudaFuncSetAttribute(reduce_splits_bulk_kernel<T, V, true>,
                                            cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kReduceBulkSmem));
        attr_set = true;
      }
      auto kern = cg ? reduce_splits_bulk_kernel<T, V, true> : reduce_splits_bulk_kernel<T, V, false>;
      QES_CUDA_CHECK(qes_launch_pdl(kern, dim3(grid), dim3(RS_THREADS), bulk_smem, st, P, nsplit, (int)cv,
                                    (const T*)partial, shift, p, y, dot_part, scal, counter, cg_done, pold, sold,
                                    counter ? (int*)(counter + 4) : (int*)nullptr));
      return QES_OK;
    }
    if (vec) {
      auto kern = cg ? reduce_splits_kernel<T, V, true, true> : reduce_splits_kernel<T, V, true, false>;
      QES_CUDA_CHECK(qes_launch_pdl(kern, dim3(grid), dim3(RS_THREADS), 0, st, P, nsplit, (int)cv, (const T*)partial,
                                    shift, p, y, dot_part, scal, counter, cg_done, pold, sold));
      return QES_OK;
    }
  }
  auto kern = cg ? reduce_splits_kernel<T, V, false, true> : reduce_splits_kernel<T, V, false, false>;
  QES_CUDA_CHECK(qes_launch_pdl(kern, dim3(grid), dim3(RS_THREADS), 0, st, P, nsplit, (int)cv, (const T*)partial, shift,
                                p, y, dot_part, scal, counter, cg_done, pold, sold));
  return QES_OK;
}

// ----------------------------------------------------------------------------
// CG state on the device (float64):
//   scal[0] rho (r^H r, or r^H D^-1 r with the Jacobi preconditioner)   scal[1] pAp
//   scal[2] rr_new = ||r||^2   scal[3] threshold^2   scal[4] done
//   scal[5] iterations   scal[6] ||b||^2   scal[7] alpha   scal[8] beta
// Partial sums are reduced by one block of 1024 threads in a fixed order.
// ----------------------------------------------------------------------------
constexpr int SC_THREADS = 1024;

__device__ __forceinline__ double block_sum_parts(int n, const double* __restrict__ parts) {
  __shared__ double red[SC_THREADS / 32];
  double v = 0.0;
  for (int q = threadIdx.x; q < n; q += blockDim.x) v += parts[q];
  v = warp_sum(v);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x == 0)
    for (int q = 0; q < (int)(blockDim.x >> 5); ++q) t += red[q];
  return t;                                // valid in thread 0
}

// dinv (optional): the Jacobi preconditioner D^-1 = 1 / diag(S + shift); the block also sums
// rho = r^H D^-1 r into rz_part (PCG's alpha / beta numerator; plain CG uses rho = r^H r)
template <class V>
__global__ void __launch_bounds__(RED_THREADS) cg_xr_kernel(int64_t P, const V* __restrict__ p, const V* __restrict__ Ap,
                                                            V* __restrict__ x, V* __restrict__ r,
                                                            double* __restrict__ scal, double* __restrict__ rr_part,
                                                            unsigned int* __restrict__ counter,
                                                            const double* __restrict__ dinv = nullptr,
                                                            double* __restrict__ rz_part = nullptr) {
  pdl_trigger();
  pdl_wait();                                              // Ap and alpha: previous kernel
  if (scal[4] != 0.0) return;                              // converged: x and r are final (every block)
  const double alpha = scal[7];
  double d = 0.0, dz = 0.0;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < P; k += (int64_t)gridDim.x * blockDim.x) {
    V rk = r[k];
    x[k] = vadd(x[k], vscale(alpha, p[k]));
    rk = vadd(rk, vscale(-alpha, Ap[k]));
    r[k] = rk;
    const double q = vdotc(rk, rk);
    d += q;
    if (dinv) dz += q * dinv[k];
  }
  __shared__ double red[RED_THREADS / 32], redz[RED_THREADS / 32];
  d = warp_sum(d);
  dz = warp_sum(dz);
  if ((threadIdx.x & 31) == 0) {
    red[threadIdx.x >> 5] = d;
    redz[threadIdx.x >> 5] = dz;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0, sz = 0;
    for (int q = 0; q < RED_THREADS / 32; ++q) {
      s += red[q];
      sz += redz[q];
    }
    rr_part[blockIdx.x] = s;
    if (dinv) rz_part[blockIdx.x] = sz;
  }
  // the last block to finish: rr_new, convergence, beta = rr_new / rr, rr <- rr_new
  __shared__ bool last;
  if (threadIdx.x == 0) {            // only thread 0 wrote this block's partial
    __threadfence();
    last = (atomicAdd(counter, 1u) == gridDim.x - 1);
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  double v = 0.0, vz = 0.0;
  for (int q = threadIdx.x; q < (int)gridDim.x; q += blockDim.x) {
    v += ((volatile double*)rr_part)[q];
    if (dinv) vz += ((volatile double*)rz_part)[q];
  }
  v = warp_sum(v);
  vz = warp_sum(vz);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) {
    red[threadIdx.x >> 5] = v;
    redz[threadIdx.x >> 5] = vz;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double rr_new = 0.0, rz_new = 0.0;
    for (int q = 0; q < RED_THREADS / 32; ++q) {
      rr_new += red[q];
      rz_new += redz[q];
    }
    const double rho_new = dinv ? rz_new : rr_new;
    if (scal[4] == 0.0) {
      scal[2] = rr_new;
      scal[5] += 1.0;
      scal[8] = (scal[0] > 0.0) ? rho_new / scal[0] : 0.0;
      scal[0] = rho_new;
      if (rr_new <= scal[3]) scal[4] = 1.0;
    }
    *counter = 0u;
  }
}

// p = r + beta p; on the tensor-core path also rewrite the V' operand tiles of the new p
template <class V>
__global__ void __launch_bounds__(RED_THREADS) cg_p_kernel(int64_t P, const V* __restrict__ r, V* __restrict__ p,
                                                           const double* __restrict__ scal, TcDims td,
                                                           uint16_t* __restrict__ vp,
                                                           const double* __restrict__ dinv = nullptr) {
  pdl_trigger();
  pdl_wait();                                              // r and beta: previous kernel
  if (scal[4] != 0.0) return;
  const double beta = scal[8];
  const int ns = td.ns, nh = td.nh;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < P; k += (int64_t)gridDim.x * blockDim.x) {
    const V zk = dinv ? vscale(dinv[k], r[k]) : r[k];     // z = D^-1 r (PCG) or r
    const V pk = vadd(zk, vscale(beta, p[k]));
    p[k] = pk;
    if (vp && k >= ns) {
      const int64_t q = k - ns;
      if (q < nh) {
        tc_put_vp_elem(td, vp, ns, (int)q, pk);                          // v_b row
      } else {
        const uint32_t qw = (uint32_t)(q - nh);                          // ns * nh < 2^32 on this path
        tc_put_vp_elem(td, vp, (int)(qw / (uint32_t)nh), (int)(qw % (uint32_t)nh), pk);
      }
    }
  }
}

// Chronopoulos-Gear CG step k, second half (one reduction per step: the split reduction of A r_k
// also sums |r_k|^2 and its last block forms alpha_k, beta_k and the convergence test):
//   p_k = r_k + beta_k p_{k-1},  s_k = A r_k + beta_k s_{k-1}  (= A p_k),
//   x_{k+1} = x_k + alpha_k p_k,  r_{k+1} = r_k - alpha_k s_k,
// and the tensor-core operand tiles of r_{k+1}, the next matvec input (Chronopoulos and Gear,
// J. Comput. Appl. Math. 25 (1989) 153-168).  beta_0 = 0: p_0 = r_0 and s_0 = A r_0 exactly.
template <class V>
__global__ void __launch_bounds__(RED_THREADS) cg_cgstep_kernel(int64_t P, const V* __restrict__ Ar,
                                                                V* __restrict__ x, V* __restrict__ r,
                                                                V* __restrict__ p, V* __restrict__ sv,
                                                                const double* __restrict__ scal, TcDims td,
                                                                uint16_t* __restrict__ vp) {
  pdl_trigger();
  pdl_wait();                                              // A r_k, alpha_k, beta_k: previous kernel
  if (scal[4] != 0.0) return;                              // converged: x is final
  const double alpha = scal[7], beta = scal[8];
  const int ns = td.ns, nh = td.nh;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < P; k += (int64_t)gridDim.x * blockDim.x) {
    const V rk = r[k], wk = Ar[k];
    const V pk = beta != 0.0 ? vadd(rk, vscale(beta, p[k])) : rk;
    const V sk = beta != 0.0 ? vadd(wk, vscale(beta, sv[k])) : wk;
    p[k] = pk;
    sv[k] = sk;
    x[k] = vadd(x[k], vscale(alpha, pk));
    const V rn = vadd(rk, vscale(-alpha, sk));
    r[k] = rn;
    if (vp && k >= ns) {
      const int64_t q = k - ns;
      if (q < nh) {
        tc_put_vp_elem(td, vp, ns, (int)q, rn);                          // v_b row
      } else {
        const uint32_t qw = (uint32_t)(q - nh);                          // ns * nh < 2^32 on this path
        tc_put_vp_elem(td, vp, (int)(qw / (uint32_t)nh), (int)(qw % (uint32_t)nh), rn);
      }
    }
  }
}

// grid of the per-iteration vector kernels: one element per thread up to RED_BLOCKS blocks (fewer
// blocks, fewer tickets on the last-block counter for small parameter vectors)
static int vec_blocks(int64_t n) {
  return (int)std::min<int64_t>(RED_BLOCKS, std::max<int64_t>(1, (n + RED_THREADS - 1) / RED_THREADS));
}

// r = p = b - A x0 (x already holds x0, Ap holds A x0)
// (p = D^-1 r with the Jacobi preconditioner dinv)
template <class V>
__global__ void cg_init_x0_kernel(int64_t P, const V* __restrict__ b, const V* __restrict__ Ax0, V* __restrict__ r,
                                  V* __restrict__ p, const double* __restrict__ dinv = nullptr) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < P; k += (int64_t)gridDim.x * blockDim.x) {
    const V rk = vadd(b[k], vscale(-1.0, Ax0[k]));
    r[k] = rk;
    p[k] = dinv ? vscale(dinv[k], rk) : rk;
  }
}

// x = 0, r = b, p = b (or D^-1 b)
template <class V>
__global__ void cg_init_kernel(int64_t P, const V* __restrict__ b, V* __restrict__ x, V* __restrict__ r,
                               V* __restrict__ p, const double* __restrict__ dinv = nullptr) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < P; k += (int64_t)gridDim.x * blockDim.x) {
    x[k] = vzero(V());
    r[k] = b[k];
    p[k] = dinv ? vscale(dinv[k], b[k]) : b[k];
  }
}

// per-block partial sums of r^H D^-1 r
template <class V>
__global__ void __launch_bounds__(RED_THREADS) wnorm2_kernel(int64_t P, const V* __restrict__ r,
                                                             const double* __restrict__ dinv,
                                                             double* __restrict__ part) {
  double d = 0.0;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < P; k += (int64_t)gridDim.x * blockDim.x)
    d += vdotc(r[k], r[k]) * dinv[k];
  __shared__ double red[RED_THREADS / 32];
  d = warp_sum(d);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = d;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0;
    for (int q = 0; q < RED_THREADS / 32; ++q) t += red[q];
    part[blockIdx.x] = t;
  }
}

// Jacobi preconditioner of S + shift: diag(S)_k = sum_s p_s |O_sk - Obar_k|^2 / Ns = mean|O_k|^2 - |Obar_k|^2
// with mean|O_k|^2 = 1 for the visible biases (sigma^2 = 1) and mean|t_m|^2 for b_m and W_im.
// Partial column sums of p_s |t_sm|^2 over sample splits (grid.y), then their fixed-order sum.
constexpr int TSQ_SPLITS = 128;
template <class T>
__global__ void tsq_part_kernel(int nh, int64_t n, const T* __restrict__ tt, const float* __restrict__ wts,
                                double* __restrict__ part) {
  const int m = blockIdx.x * 32 + threadIdx.x;
  const int64_t s0 = (int64_t)blockIdx.y * n / gridDim.y, s1 = (int64_t)(blockIdx.y + 1) * n / gridDim.y;
  double acc = 0.0;
  if (m < nh)
    for (int64_t s = s0 + threadIdx.y; s < s1; s += blockDim.y) {
      const T t = tt[s * nh + m];
      double a;
      if constexpr (ScalarTraits<T>::is_complex) a = (double)t.x * t.x + (double)t.y * t.y;
      else a = (double)t * t;
      acc += wts ? (double)wts[s] * a : a;
    }
  __shared__ double red[8][32];
  red[threadIdx.y][threadIdx.x] = acc;
  __syncthreads();
  if (threadIdx.y == 0 && m < nh) {
    double t = 0.0;
    for (int q = 0; q < (int)blockDim.y; ++q) t += red[q][threadIdx.x];
    part[(int64_t)blockIdx.y * nh + m] = t;
  }
}
__global__ void tsq_sum_kernel(int nh, int nsplit, double inv_n, const double* __restrict__ part,
                               double* __restrict__ tsq) {
  for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < nh; m += gridDim.x * blockDim.x) {
    double t = 0.0;
    for (int z = 0; z < nsplit; ++z) t += part[(int64_t)z * nh + m];
    tsq[m] = t * inv_n;
  }
}
// obar_h = O^H p / Ns (the conjugated weighted mean of the O rows); dinv = 1 / (max(diag S, 0) + shift)
template <class V>
__global__ void jacobi_dinv_kernel(int ns, int nh, int64_t P, const double* __restrict__ tsq,
                                   const V* __restrict__ obar_h, double shift, double* __restrict__ dinv) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < P; k += (int64_t)gridDim.x * blockDim.x) {
    double msq = 1.0;
    if (k >= ns) msq = tsq[(k < ns + nh) ? (int)(k - ns) : (int)((k - ns - nh) % nh)];
    const double d = fmax(msq - vdotc(obar_h[k], obar_h[k]), 0.0) + shift;
    dinv[k] = d > 0.0 ? 1.0 / d : 1.0;
  }
}
__global__ void fill_ones_kernel(int64_t n, float2* __restrict__ g) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x)
    g[k] = make_float2(1.f, 0.f);
}

// parts_r: dot partials of ||r0||^2 for a start x0 != 0 (nullptr: r0 = b)
// parts_z: dot partials of r0^H D^-1 r0 (Jacobi PCG: rho0; nullptr: rho0 = ||r0||^2)
__global__ void __launch_bounds__(SC_THREADS) cg_setup_kernel(int n, const double* __restrict__ parts, double rtol,
                                                              double atol, double* __restrict__ scal,
                                                              const double* __restrict__ parts_r = nullptr,
                                                              const double* __restrict__ parts_z = nullptr) {
  const double s = block_sum_parts(n, parts);
  double rr0 = s;
  if (parts_r) {
    __syncthreads();                                      // block_sum_parts reuses its shared buffer
    rr0 = block_sum_parts(n, parts_r);
  }
  double rho0 = rr0;
  if (parts_z) {
    __syncthreads();
    rho0 = block_sum_parts(n, parts_z);
  }
  if (threadIdx.x != 0) return;
  scal[0] = rho0;                   // rho = ||r0||^2 (CG) or r0^H D^-1 r0 (PCG)
  scal[6] = s;                      // ||b||^2
  const double th = fmax(rtol * sqrt(s), atol);
  scal[3] = th * th;
  scal[5] = 0.0;
  scal[4] = (rr0 <= scal[3]) ? 1.0 : 0.0;
  scal[1] = 0.0;
  scal[2] = rr0;
  scal[7] = 0.0;
  scal[8] = 0.0;
  scal[9] = 0.0;
}

template <class V>
__global__ void __launch_bounds__(RED_THREADS) norm2_kernel(int64_t P, const V* __restrict__ b, double* __restrict__ part) {
  double d = 0.0;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < P; k += (int64_t)gridDim.x * blockDim.x)
    d += vdotc(b[k], b[k]);
  __shared__ double red[RED_THREADS / 32];
  d = warp_sum(d);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = d;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0;
    for (int q = 0; q < RED_THREADS / 32; ++q) s += red[q];
    part[blockIdx.x] = s;
  }
}

// ||b - y||^2: per-block partial sums, then one block adds them into *out
template <class V>
__global__ void __launch_bounds__(RED_THREADS) diff_norm2_kernel(int64_t P, const V* __restrict__ b,
                                                                 const V* __restrict__ y, double* __restrict__ part) {
  double d = 0.0;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < P; k += (int64_t)gridDim.x * blockDim.x) {
    const V e = vadd(b[k], vscale(-1.0, y[k]));
    d += vdotc(e, e);
  }
  __shared__ double red[RED_THREADS / 32];
  d = warp_sum(d);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = d;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0;
    for (int q = 0; q < RED_THREADS / 32; ++q) t += red[q];
    part[blockIdx.x] = t;
  }
}
__global__ void __launch_bounds__(SC_THREADS) sum_parts_kernel(int n, const double* __restrict__ parts,
                                                               double* __restrict__ out) {
  const double t = block_sum_parts(n, parts);
  if (threadIdx.x == 0) *out = t;
}

template <class V>
__global__ void scale_vec_kernel(int64_t P, double s, V* __restrict__ x) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < P; k += (int64_t)gridDim.x * blockDim.x)
    x[k] = vscale(s, x[k]);
}

// ----------------------------------------------------------------------------
// One kernel for the vector part of a CG iteration: Ap = sum of the split
// partials + shift p (pAp), alpha; x += alpha p, r -= alpha Ap (rr_new), beta;
// p = r + beta p (+ the V' tiles of the tensor-core path).  The two global
// dependencies are grid barriers of a cooperative launch (all CTAs resident);
// each barrier wait is bounded and records a time-out in *err.
// ----------------------------------------------------------------------------
constexpr int CF_TX = 32, CF_TY = 16;            // 512 threads: 32 columns x 16 split groups

// count and gen live in different 128-byte lines; waiters poll gen with plain volatile loads so
// that the arrivals (atomics on count) do not queue behind polling atomics.  BarCfg (sr_tc.h) is the
// test hook set by qes_sr_set_barrier_test.

__device__ __forceinline__ void grid_barrier(unsigned int* count, unsigned int* gen, unsigned int nb, int* err,
                                             BarCfg bc) {
  nb += bc.extra;
  __syncthreads();
  if (threadIdx.x == 0 && threadIdx.y == 0) {
    volatile unsigned int* vgen = gen;
    const unsigned int g = *vgen;
    __threadfence();
    if (atomicAdd(count, 1u) == nb - 1) {
      *count = 0u;
      __threadfence();
      atomicAdd(gen, 1u);
    } else {
      uint32_t it = 0;
      while (*vgen == g) {
        if (++it > bc.limit) { atomicExch(err, 1); break; }
        __nanosleep(20);
      }
    }
    __threadfence();
  }
  __syncthreads();
}

// x/r update and direction update of a CG step in one launch (qes_set_cg_xrp): phase 1 as
// cg_xr_kernel (x += alpha p, r -= alpha Ap, per-block |r|^2 and r^H D^-1 r partials), a bounded
// grid barrier, then every CTA sums the grid's partials in the same fixed order as cg_xr_kernel's
// last block (so the scalars are bit-identical to the two-kernel form) and updates its own slice of
// p and the operand tiles.  One launch boundary and one last-block step fewer per iteration.  The
// grid (<= 296 blocks of 256 threads) is co-resident once every CTA has executed the programmatic
// trigger, which is what lets the next kernel launch, so the barrier cannot wait on a CTA that a
// dependent kernel keeps off the SMs; a barrier wait that runs out sets *err (the solve reports
// QES_ERR_TIMEOUT).
template <class V>
__global__ void __launch_bounds__(RED_THREADS) cg_xrp_kernel(int64_t P, const V* __restrict__ Ap, V* __restrict__ x,
                                                             V* __restrict__ r, V* __restrict__ p,
                                                             double* __restrict__ scal, double* __restrict__ part,
                                                             unsigned int* __restrict__ bar, int* __restrict__ err,
                                                             TcDims td, uint16_t* __restrict__ vp, BarCfg bc,
                                                             const double* __restrict__ dinv) {
  pdl_trigger();
  pdl_wait();                                              // Ap and alpha: previous kernel
  // every CTA reads the scalars before any CTA can pass the barrier (CTA 0 rewrites them after it)
  const double rho = scal[0], thresh = scal[3], alpha = scal[7];
  if (scal[4] != 0.0) return;                              // converged at an earlier step
  const unsigned int nb = gridDim.x;
  const int tid = threadIdx.x;
  __shared__ double sred[RED_THREADS / 32];
  auto block_sum = [&](double v) -> double {
    v = warp_sum(v);
    if ((tid & 31) == 0) sred[tid >> 5] = v;
    __syncthreads();
    double t = 0.0;
    for (int q = 0; q < RED_THREADS / 32; ++q) t += sred[q];
    __syncthreads();
    return t;
  };
  double e = 0.0, ez = 0.0;
  const int64_t stride = (int64_t)nb * RED_THREADS;
  for (int64_t k = (int64_t)blockIdx.x * RED_THREADS + tid; k < P; k += stride) {
    x[k] = vadd(x[k], vscale(alpha, p[k]));
    const V rk = vadd(r[k], vscale(-alpha, Ap[k]));
    r[k] = rk;
    const double q = vdotc(rk, rk);
    e += q;
    if (dinv) ez += q * dinv[k];
  }
  e = block_sum(e);
  if (tid == 0) part[blockIdx.x] = e;
  if (dinv) {
    ez = block_sum(ez);
    if (tid == 0) part[nb + blockIdx.x] = ez;
  }
  grid_barrier(bar, bar + 32, nb, err, bc);
  auto sum_parts = [&](const double* src) -> double {
    double v = 0.0;
    for (unsigned int b = tid; b < nb; b += RED_THREADS) v += __ldcg(src + b);
    return block_sum(v);
  };
  const double rr_new = sum_parts(part);
  const double rho_new = dinv ? sum_parts(part + nb) : rr_new;
  const double beta = (rho > 0.0) ? rho_new / rho : 0.0;
  const bool conv = rr_new <= thresh;
  if (!conv) {
    const int ns = td.ns, nh = td.nh;
    for (int64_t k = (int64_t)blockIdx.x * RED_THREADS + tid; k < P; k += stride) {
      const V zk = dinv ? vscale(dinv[k], r[k]) : r[k];
      const V pk = vadd(zk, vscale(beta, p[k]));
      p[k] = pk;
      if (vp && k >= ns) {
        const int64_t q = k - ns;
        if (q < nh) {
          tc_put_vp_elem(td, vp, ns, (int)q, pk);                        // v_b row
        } else {
          const uint32_t qw = (uint32_t)(q - nh);                        // ns * nh < 2^32 on this path
          tc_put_vp_elem(td, vp, (int)(qw / (uint32_t)nh), (int)(qw % (uint32_t)nh), pk);
        }
      }
    }
  }
  if (blockIdx.x == 0 && tid == 0) {
    scal[2] = rr_new;
    scal[5] += 1.0;
    scal[8] = beta;
    scal[0] = rho_new;
    if (conv) scal[4] = 1.0;
  }
}

// cv: column vectors per block pass (16-byte vectors when VEC), chosen by the host like the
// standalone split reduction (every thread issues its split loads in one batch)
template <class T, class V, bool VEC>
__global__ void __launch_bounds__(CF_TX * CF_TY) cg_fused_kernel(int64_t P, int nsplit, int cv,
                                                                 const T* __restrict__ partial,
                                                                 double shift, V* __restrict__ x, V* __restrict__ r,
                                                                 V* __restrict__ p, V* __restrict__ Ap,
                                                                 double* __restrict__ scal, double* __restrict__ part,
                                                                 unsigned int* __restrict__ bar, int* __restrict__ err,
                                                                 TcDims td, uint16_t* __restrict__ vp, BarCfg bc,
                                                                 const double* __restrict__ dinv) {
  // launched by programmatic dependent launch (qes_set_cg_fused_pdl) the grid is co-resident once
  // every CTA has run the trigger (the next kernel launches only then); cooperative launches see
  // both calls as no-ops
  pdl_trigger();
  pdl_wait();                                      // the split partials and the CG scalars
  const double rr = scal[0], thresh = scal[3];     // rr: rho (r^H D^-1 r with the preconditioner)
  if (scal[4] != 0.0) return;                      // converged: every CTA leaves (scal only changes below)
  if (*(volatile int*)err != 0) return;            // an earlier barrier wait gave up: the solve is abandoned
  constexpr int NT = CF_TX * CF_TY;
  constexpr int E = VEC ? (int)(16 / sizeof(T)) : 1;      // columns per vector
  const int tid = threadIdx.y * CF_TX + threadIdx.x;
  const unsigned int nb = gridDim.x;
  __shared__ V red[NT * E];                                // [split group][column vector][E]
  __shared__ double sred[NT / 32];
  // phase 1: Ap and p^H Ap (the split reduction of reduce_splits_kernel)
  double d = 0.0;
  {
    const int groups = NT / cv, c = tid % cv, sg = tid / cv;
    const int64_t nvec = P / E;
    for (int64_t v0 = (int64_t)blockIdx.x * cv; v0 < nvec; v0 += (int64_t)nb * cv) {
      const int64_t vi = v0 + c;
      V g[E];
#pragma unroll
      for (int e = 0; e < E; ++e) g[e] = vzero(V());
      if (sg < groups && vi < nvec) {
        for (int z0 = sg; z0 < nsplit; z0 += groups * RS_BATCH) {
          if constexpr (VEC) {
            float4 q[RS_BATCH];
            const float4* src = reinterpret_cast<const float4*>(partial) + vi;
#pragma unroll
            for (int b = 0; b < RS_BATCH; ++b) {
              const int z = z0 + b * groups;
              q[b] = (z < nsplit) ? __ldcg(src + (int64_t)z * nvec) : make_float4(0.f, 0.f, 0.f, 0.f);
            }
#pragma unroll
            for (int b = 0; b < RS_BATCH; ++b) acc4(g, q[b]);
          } else {
            T q[RS_BATCH];
#pragma unroll
            for (int b = 0; b < RS_BATCH; ++b) {
              const int z = z0 + b * groups;
              q[b] = (z < nsplit) ? partial[(int64_t)z * P + vi] : T{};
            }
#pragma unroll
            for (int b = 0; b < RS_BATCH; ++b) g[0] = vadd(g[0], to_d(q[b]));
          }
        }
      }
      if (sg < groups) {
#pragma unroll
        for (int e = 0; e < E; ++e) red[(sg * cv + c) * E + e] = g[e];
      }
      __syncthreads();
      if (tid < cv * E) {
        const int64_t kk = v0 * E + tid;
        if (kk < P) {
          V t = red[tid];
          for (int q = 1; q < groups; ++q) t = vadd(t, red[q * cv * E + tid]);
          const V pk = p[kk];
          t = vadd(t, vscale(shift, pk));
          Ap[kk] = t;
          d += vdotc(pk, t);
        }
      }
      __syncthreads();
    }
  }
  auto block_sum = [&](double v) -> double {
    v = warp_sum(v);
    if ((tid & 31) == 0) sred[tid >> 5] = v;
    __syncthreads();
    double t = 0.0;
    for (int q = 0; q < CF_TX * CF_TY / 32; ++q) t += sred[q];
    __syncthreads();
    return t;
  };
  d = block_sum(d);
  if (tid == 0) part[blockIdx.x] = d;
  grid_barrier(bar, bar + 32, nb, err, bc);
  // every CTA sums the nb partials with the whole block (same fixed order in every CTA)
  auto sum_parts = [&](const double* src) -> double {
    double v = 0.0;
    for (unsigned int b = tid; b < nb; b += CF_TX * CF_TY) v += __ldcg(src + b);
    return block_sum(v);
  };
  const double pap = sum_parts(part);
  const double alpha = (pap > 0.0) ? rr / pap : 0.0;
  // phase 2: x, r, r^H r (and r^H D^-1 r)
  double e = 0.0, ez = 0.0;
  const int64_t stride = (int64_t)nb * NT;
  for (int64_t k = (int64_t)blockIdx.x * NT + tid; k < P; k += stride) {
    x[k] = vadd(x[k], vscale(alpha, p[k]));
    const V rk = vadd(r[k], vscale(-alpha, Ap[k]));
    r[k] = rk;
    const double q = vdotc(rk, rk);
    e += q;
    if (dinv) ez += q * dinv[k];
  }
  e = block_sum(e);
  if (tid == 0) part[nb + blockIdx.x] = e;
  if (dinv) {
    ez = block_sum(ez);
    if (tid == 0) part[2 * nb + blockIdx.x] = ez;
  }
  grid_barrier(bar, bar + 32, nb, err, bc);
  const double rr_new = sum_parts(part + nb);
  const double rho_new = dinv ? sum_parts(part + 2 * nb) : rr_new;
  const double beta = (rr > 0.0) ? rho_new / rr : 0.0;
  const bool conv = rr_new <= thresh;
  // phase 3: direction update (same index map as phase 2: each thread updates what it wrote)
  if (!conv) {
    const int ns = td.ns, nh = td.nh;
    for (int64_t k = (int64_t)blockIdx.x * NT + tid; k < P; k += stride) {
      const V zk = dinv ? vscale(dinv[k], r[k]) : r[k];
      const V pk = vadd(zk, vscale(beta, p[k]));
      p[k] = pk;
      if (vp && k >= ns) {
        const int64_t q = k - ns;
        if (q < nh) tc_put_vp_elem(td, vp, ns, (int)q, pk);
        else tc_put_vp_elem(td, vp, (int)((q - nh) / nh), (int)((q - nh) % nh), pk);
      }
    }
  }
  if (blockIdx.x == 0 && tid == 0) {
    scal[1] = pap; scal[7] = alpha; scal[2] = rr_new; scal[8] = beta; scal[0] = rho_new;
    scal[5] += 1.0;
    if (conv) scal[4] = 1.0;
  }
}

// ----------------------------------------------------------------------------
// MINRES (Paige & Saunders 1975, the recurrences of SciPy's minres without a
// preconditioner) on the Hermitian S + shift.  The Lanczos vector v is the
// matvec input (the CG's p buffer, V' tiles on the tensor-core path), y = A v
// comes out of the split reduction with alpha = v^H A v (its dot partials, the
// last block's pAp = scal[1]).  State scalars in ms[]:
//   0 beta   1 oldb   2 dbar   3 epsln   4 phibar   5 cs   6 sn   7 phi
//   8 delta  9 denom 10 oldeps 11 converged 12 gmax 13 gmin
// and the shared flags of the CG: scal[2] = phibar^2 (the residual estimate),
// scal[3] threshold^2, scal[4] done, scal[5] iterations, scal[6] ||b||^2.
// ----------------------------------------------------------------------------
// r2 = r1 = b - A x0 (x0 given: Ax0 in y) or b; partial sums of ||r2||^2
template <class V>
__global__ void minres_init_kernel(int64_t P, const V* __restrict__ b, const V* __restrict__ Ax0, V* __restrict__ x,
                                   V* __restrict__ r1, V* __restrict__ r2, V* __restrict__ w1, V* __restrict__ w2,
                                   bool has_x0) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < P; k += (int64_t)gridDim.x * blockDim.x) {
    const V rk = has_x0 ? vadd(b[k], vscale(-1.0, Ax0[k])) : b[k];
    if (!has_x0) x[k] = vzero(V());
    r1[k] = rk;
    r2[k] = rk;
    w1[k] = vzero(V());
    w2[k] = vzero(V());
  }
}
// parts: ||b||^2 partials, parts_r: ||r0||^2 partials
__global__ void __launch_bounds__(SC_THREADS) minres_setup_kernel(int n, const double* __restrict__ parts,
                                                                  const double* __restrict__ parts_r, double rtol,
                                                                  double atol, double* __restrict__ scal,
                                                                  double* __restrict__ ms) {
  const double bb = block_sum_parts(n, parts);
  __syncthreads();
  const double rr0 = block_sum_parts(n, parts_r);
  if (threadIdx.x != 0) return;
  const double beta1 = sqrt(rr0);
  scal[6] = bb;
  const double th = fmax(rtol * sqrt(bb), atol);
  scal[3] = th * th;
  scal[2] = rr0;
  scal[5] = 0.0;
  scal[4] = (rr0 <= scal[3]) ? 1.0 : 0.0;
  for (int q = 0; q < 32; ++q) ms[q] = 0.0;
  ms[0] = beta1;                  // beta
  ms[4] = beta1;                  // phibar
  ms[5] = -1.0;                   // cs
  ms[12] = 0.0;                   // gmax
  ms[13] = 1e308;                 // gmin
}
// v = r2 / beta (the first Lanczos vector; later ones come from minres_update_kernel)
template <class V>
__global__ void minres_v_kernel(int64_t P, const V* __restrict__ r2, V* __restrict__ v, const double* __restrict__ ms,
                                TcDims td, uint16_t* __restrict__ vp) {
  const double s = ms[0] > 0.0 ? 1.0 / ms[0] : 0.0;
  const int ns = td.ns, nh = td.nh;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < P; k += (int64_t)gridDim.x * blockDim.x) {
    const V vk = vscale(s, r2[k]);
    v[k] = vk;
    if (vp && k >= ns) {
      const int64_t q = k - ns;
      if (q < nh) tc_put_vp_elem(td, vp, ns, (int)q, vk);
      else tc_put_vp_elem(td, vp, (int)((q - nh) / nh), (int)((q - nh) % nh), vk);
    }
  }
}
// y = A v - (beta / oldb) r1 - (alpha / beta) r2;  r1 <- r2;  r2 <- y;  ||y||^2.  The last block runs the
// scalar recurrences: beta_new = ||y||, the Givens rotation that updates the QR factor of the Lanczos
// tridiagonal, phi / phibar (phibar = the residual norm of the iterate), the convergence test.
template <class V>
__global__ void __launch_bounds__(RED_THREADS) minres_lanczos_kernel(int64_t P, const V* __restrict__ Av,
                                                                     V* __restrict__ r1, V* __restrict__ r2,
                                                                     double* __restrict__ scal, double* __restrict__ ms,
                                                                     double* __restrict__ part,
                                                                     unsigned int* __restrict__ counter) {
  pdl_trigger();
  pdl_wait();                                              // A v and alpha: previous kernel
  if (scal[4] != 0.0) return;
  const double beta = ms[0], oldb = ms[1], alpha = scal[1];
  const double c1 = oldb > 0.0 ? beta / oldb : 0.0, c2 = beta > 0.0 ? alpha / beta : 0.0;
  double d = 0.0;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < P; k += (int64_t)gridDim.x * blockDim.x) {
    const V r2k = r2[k];
    const V y = vadd(vadd(Av[k], vscale(-c1, r1[k])), vscale(-c2, r2k));
    r1[k] = r2k;
    r2[k] = y;
    d += vdotc(y, y);
  }
  __shared__ double red[RED_THREADS / 32];
  __shared__ bool last;
  d = warp_sum(d);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = d;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int q = 0; q < RED_THREADS / 32; ++q) t += red[q];
    part[blockIdx.x] = t;
    __threadfence();
    last = (atomicAdd(counter, 1u) == gridDim.x - 1);
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  double v = 0.0;
  for (int q = threadIdx.x; q < (int)gridDim.x; q += blockDim.x) v += ((volatile double*)part)[q];
  v = warp_sum(v);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double yy = 0.0;
    for (int q = 0; q < RED_THREADS / 32; ++q) yy += red[q];
    const double bnew = sqrt(yy);
    const double cs = ms[5], sn = ms[6], dbar = ms[2];
    const double oldeps = ms[3];
    const double delta = cs * dbar + sn * alpha;
    const double gbar = sn * dbar - cs * alpha;
    const double epsln = sn * bnew;
    const double dbar_new = -cs * bnew;
    const double gamma = fmax(hypot(gbar, bnew), 1e-300);
    const double cs_new = gbar / gamma, sn_new = bnew / gamma;
    const double phi = cs_new * ms[4];
    const double phibar = sn_new * ms[4];
    ms[1] = beta;  ms[0] = bnew;  ms[2] = dbar_new;  ms[3] = epsln;  ms[4] = phibar;
    ms[5] = cs_new;  ms[6] = sn_new;  ms[7] = phi;  ms[8] = delta;  ms[9] = 1.0 / gamma;  ms[10] = oldeps;
    ms[12] = fmax(ms[12], gamma);
    ms[13] = fmin(ms[13], gamma);
    scal[2] = phibar * phibar;
    ms[11] = (phibar * phibar <= scal[3] || bnew == 0.0) ? 1.0 : 0.0;
    *counter = 0u;
  }
}
// w = (v - oldeps w_(k-2) - delta w_(k-1)) / gamma;  x += phi w;  v <- r2 / beta_new (+ its V' tiles); the
// last block counts the iteration and publishes the convergence found by the Lanczos step
template <class V>
__global__ void __launch_bounds__(RED_THREADS) minres_update_kernel(int64_t P, V* __restrict__ v, V* __restrict__ w1,
                                                                    V* __restrict__ w2, V* __restrict__ x,
                                                                    const V* __restrict__ r2, double* __restrict__ scal,
                                                                    const double* __restrict__ ms,
                                                                    unsigned int* __restrict__ counter, TcDims td,
                                                                    uint16_t* __restrict__ vp) {
  pdl_trigger();
  pdl_wait();
  if (scal[4] != 0.0) return;
  const double oldeps = ms[10], delta = ms[8], denom = ms[9], phi = ms[7];
  const double s = ms[0] > 0.0 ? 1.0 / ms[0] : 0.0;
  const bool conv = ms[11] != 0.0;
  const int ns = td.ns, nh = td.nh;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < P; k += (int64_t)gridDim.x * blockDim.x) {
    const V wk = vscale(denom, vadd(vadd(v[k], vscale(-oldeps, w1[k])), vscale(-delta, w2[k])));
    w1[k] = w2[k];
    w2[k] = wk;
    x[k] = vadd(x[k], vscale(phi, wk));
    if (!conv) {
      const V vk = vscale(s, r2[k]);
      v[k] = vk;
      if (vp && k >= ns) {
        const int64_t q = k - ns;
        if (q < nh) tc_put_vp_elem(td, vp, ns, (int)q, vk);
        else tc_put_vp_elem(td, vp, (int)((q - nh) / nh), (int)((q - nh) % nh), vk);
      }
    }
  }
  __shared__ bool last;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    last = (atomicAdd(counter, 1u) == gridDim.x - 1);
  }
  __syncthreads();
  if (!last || threadIdx.x != 0) return;
  __threadfence();
  scal[5] += 1.0;
  if (conv) scal[4] = 1.0;
  *counter = 0u;
}

// ----------------------------------------------------------------------------
// workspace layout
// ----------------------------------------------------------------------------
struct SRWork {
  float2* w;          // [Ns]
  float2* wpart;      // [ceil(nh / PT_U)][Ns] unit-block partials of w (plain form)
  const float* wts;   // per-sample weights normalised to sum Ns, or nullptr (uniform); set per call
  bool fp64;          // float64 contractions on CUDA cores (impl 3): partials, wpart and w64 in float64
  double2* w64;       // [Ns] O v of the float64 form
  double* wmean;      // [2] (+ pad)
  void* partial;      // [nsplit][P] of T
  void* x; void* r; void* p; void* Ap; void* b;   // [P] of V each
  double* parts;      // [RED_BLOCKS]
  double* scal;       // [16]
  double* dinv;       // [P] Jacobi preconditioner 1 / diag(S + shift)
  void* mr2; void* mw1; void* mw2;   // [P] of V each: MINRES r2, w_(k-2), w_(k-1)
  double* mscal;      // [32] MINRES recurrence scalars
  double* tsq;        // [nh] weighted mean of |t_m|^2, then [TSQ_SPLITS][nh] partial sums
  unsigned int* counter;  // [2] last-block tickets (reduce, x/r update)
  bool tc;            // tensor-core matvec in use
  TcDims td;
  TcWork tw;
  int nsplit;         // partial P-vectors written by the O^H u stage
  int mv_nsplit;      // partial P-vectors written by the matvec (tc_matvec_nsplit on the tensor-core path)
  size_t total;
};

static size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

static SRWork sr_layout(int dtype, int ns, int nh, int64_t n_samples, char* base) {
  const int64_t P = (int64_t)ns + nh + (int64_t)ns * nh;
  const size_t ts = (dtype == QES_DTYPE_C64) ? sizeof(float2) : sizeof(float);
  const size_t vs = (dtype == QES_DTYPE_C64) ? sizeof(double2) : sizeof(double);
  const int64_t nsplit_simt = (n_samples + PT_SPLIT - 1) / PT_SPLIT;
  SRWork L;
  L.td = TcDims{};
  const bool tc_ok = tc_plan(dtype, ns, nh, n_samples, &L.td);
  const int impl = g_sr_impl.load();
  L.fp64 = impl == 3;
  L.tc = tc_ok && impl != 1 && !L.fp64;
  const int64_t nsplit_max = std::max<int64_t>(nsplit_simt, tc_ok ? std::max(L.td.nsplit, tc_matvec_nsplit(L.td)) : 1);
  L.nsplit = (int)(L.tc ? L.td.nsplit : nsplit_simt);
  L.mv_nsplit = (int)(L.tc ? tc_matvec_nsplit(L.td) : nsplit_simt);
  size_t off = 0;
  auto take = [&](size_t bytes) { char* p = base ? base + off : nullptr; off += align256(bytes); return p; };
  L.w = (float2*)take((size_t)n_samples * sizeof(float2));
  L.wpart = (float2*)take((size_t)((nh + PT_U - 1) / PT_U) * n_samples * (L.fp64 ? sizeof(double2) : sizeof(float2)));
  L.w64 = L.fp64 ? (double2*)take((size_t)n_samples * sizeof(double2)) : nullptr;
  L.wmean = (double*)take(4 * sizeof(double));
  L.partial = take((size_t)std::max<int64_t>(nsplit_max, 1) * P * (L.fp64 ? vs : ts));
  L.x = take(P * vs); L.r = take(P * vs); L.p = take(P * vs); L.Ap = take(P * vs); L.b = take(P * vs);
  L.parts = (double*)take(5 * std::max(RED_BLOCKS, RS_MAX_BLOCKS) * sizeof(double));
  L.scal = (double*)take(16 * sizeof(double));
  L.dinv = (double*)take(P * sizeof(double));
  L.mr2 = take(P * vs); L.mw1 = take(P * vs); L.mw2 = take(P * vs);
  L.mscal = (double*)take(32 * sizeof(double));
  L.tsq = (double*)take((size_t)(TSQ_SPLITS + 1) * nh * sizeof(double));
  L.counter = (unsigned int*)take(128 * sizeof(unsigned int));     // tickets, barrier words (own lines)
  char* tcb = tc_ok ? take(tc_workspace_bytes(L.td)) : nullptr;
  L.tw = (tc_ok && base) ? tc_layout(L.td, tcb) : TcWork{};
  L.wts = nullptr;
  L.total = off;
  return L;
}

extern "C" int qes_sr_workspace_bytes(int dtype, int ns, int nh, int64_t n_samples, size_t* bytes) {
  QES_ARG_CHECK(bytes && ns > 0 && nh > 0 && n_samples >= 0, "qes_sr_workspace_bytes: bad args");
  *bytes = sr_layout(dtype, ns, nh, n_samples, nullptr).total;
  return QES_OK;
}

// split partials of O^H (wts (w - mean(w)) * scale) on the CUDA cores (register tiles); the float64
// form (fp64) accumulates in double, from w64 when it is the form's own O v (float64), else from w
template <class T>
static int launch_ohu_plain(int ns, int nh, int64_t n_samples, const uint32_t* bits, const T* tt, const float2* w,
                            const double* wmean, double scale, void* partial, cudaStream_t st,
                            const double* cg_done = nullptr, const float* wts = nullptr, bool fp64 = false,
                            const double2* w64 = nullptr) {
  using V = typename VecT<T>::type;
  const int64_t nsplit = (n_samples + PT_SPLIT - 1) / PT_SPLIT;
  QES_ARG_CHECK(nsplit <= 65535, "SR: too many samples");
  const int R = fp64 ? 4 : pt_rows_ohu(ns);
  dim3 grid((nh + 1 + PT_U - 1) / PT_U, (ns + 1 + PT_TY * R - 1) / (PT_TY * R), (unsigned)nsplit);
  const dim3 blk(PT_TX, PT_TY);
  const int pf = qes_prof_begin(QES_PROF_OHU, st);
  if (fp64) {
    if (w64)
      ohu_tile_kernel<T, V, double2, 4, PT_K64><<<grid, blk, 0, st>>>(ns, nh, n_samples, bits, tt, w64, wmean, scale,
                                                                      (V*)partial, cg_done, wts);
    else
      ohu_tile_kernel<T, V, float2, 4, PT_K64><<<grid, blk, 0, st>>>(ns, nh, n_samples, bits, tt, w, wmean, scale,
                                                                     (V*)partial, cg_done, wts);
  } else if (R == 8) {
    ohu_tile_kernel<T, T, float2, 8, PT_K><<<grid, blk, 0, st>>>(ns, nh, n_samples, bits, tt, w, wmean, scale,
                                                                 (T*)partial, cg_done, wts);
  } else {
    ohu_tile_kernel<T, T, float2, 4, PT_K><<<grid, blk, 0, st>>>(ns, nh, n_samples, bits, tt, w, wmean, scale,
                                                                 (T*)partial, cg_done, wts);
  }
  QES_LAUNCH_CHECK();
  qes_prof_end(pf, st);
  return QES_OK;
}

// g = O^H (wts (w - mean(w)) * scale)   [+ shift * p, dot partials]   into y
template <class T, class V>
static int apply_ohu(int ns, int nh, int64_t n_samples, const uint32_t* bits, const T* tt, const float2* w,
                     const double* wmean, double scale, const SRWork& L, double shift, const V* p, V* y,
                     double* dot_part, cudaStream_t st, const double* cg_done = nullptr, const V* pold = nullptr,
                     const V* sold = nullptr) {
  const int64_t P = (int64_t)ns + nh + (int64_t)ns * nh;
  const int64_t nsplit = (n_samples + PT_SPLIT - 1) / PT_SPLIT;
  const double2* w64 = (L.fp64 && w == L.w) ? L.w64 : nullptr;     // the form's own O v
  if (int rc = launch_ohu_plain<T>(ns, nh, n_samples, bits, tt, w, wmean, scale, L.partial, st, cg_done, L.wts,
                                   L.fp64, w64))
    return rc;
  const int pfr = qes_prof_begin(QES_PROF_REDUCE, st);
  if (L.fp64) {
    if (int rc_ = launch_reduce_splits<V, V>(P, (int)nsplit, L.partial, shift, p, y,
        dot_part, dot_part ? L.scal : nullptr, L.counter, st, cg_done, pold, sold)) return rc_;
  } else {
    if (int rc_ = launch_reduce_splits<T, V>(P, (int)nsplit, L.partial, shift, p, y,
        dot_part, dot_part ? L.scal : nullptr, L.counter, st, cg_done, pold, sold)) return rc_;
  }
  QES_LAUNCH_CHECK();
  qes_prof_end(pfr, st);
  return QES_OK;
}

// w = O v on the CUDA cores (register tiles; unit-block partials summed in a fixed order), and
// its float64 mean when wmean is given; the float64 form writes L.w64 instead of w
template <class T, class V>
static int apply_ov(int ns, int nh, int64_t n_samples, const uint32_t* bits, const T* tt, const V* v, float2* w,
                    double* wmean, const SRWork& L, cudaStream_t st, const double* cg_done = nullptr) {
  const int nub = (nh + PT_U - 1) / PT_U;
  const int R = L.fp64 ? 4 : pt_rows_ov(n_samples);
  dim3 grid((unsigned)((n_samples + PT_TY * R - 1) / (PT_TY * R)), (unsigned)nub);
  QES_ARG_CHECK(nub <= 65535, "SR: nh too large");
  const dim3 blk(PT_TX, PT_TY);
  const int pf = qes_prof_begin(QES_PROF_OV, st);
  if (L.fp64)
    ov_tile_kernel<T, V, V, 4, PT_K64><<<grid, blk, 0, st>>>(ns, nh, n_samples, bits, tt, v, (double2*)L.wpart,
                                                             cg_done);
  else if (R == 8)
    ov_tile_kernel<T, T, V, 8, PT_K><<<grid, blk, 0, st>>>(ns, nh, n_samples, bits, tt, v, L.wpart, cg_done);
  else
    ov_tile_kernel<T, T, V, 4, PT_K><<<grid, blk, 0, st>>>(ns, nh, n_samples, bits, tt, v, L.wpart, cg_done);
  QES_LAUNCH_CHECK();
  qes_prof_end(pf, st);
  if (L.fp64)
    wsum_kernel<double2><<<1, 1024, 0, st>>>(n_samples, nub, (const double2*)L.wpart, L.w64, wmean, cg_done, L.wts);
  else
    wsum_kernel<float2><<<1, 1024, 0, st>>>(n_samples, nub, L.wpart, w, wmean, cg_done, L.wts);
  QES_LAUNCH_CHECK();
  return QES_OK;
}

template <class T>
static int sr_force_t(int ns, int nh, int64_t n_samples, const uint32_t* bits, const T* tt, const float2* eloc,
                      typename VecT<T>::type* F, const SRWork& L, cudaStream_t st) {
  using V = typename VecT<T>::type;
  mean_c_kernel<<<1, MEAN_THREADS, 0, st>>>(n_samples, eloc, L.wmean, L.wts);
  QES_LAUNCH_CHECK();
  if (L.tc) {
    const int dtype = ScalarTraits<T>::is_complex ? QES_DTYPE_C64 : QES_DTYPE_F32;
    int rc = tc_ohu(dtype, L.td, n_samples, eloc, (const double2*)L.wmean, -1, 1.0 / (double)n_samples, L.partial,
                    L.tw, st);
    if (rc) return rc;
    const int64_t P = (int64_t)ns + nh + (int64_t)ns * nh;
    if (int rc_ = launch_reduce_splits<T, V>(P, L.nsplit, L.partial, 0.0, nullptr, F,
        nullptr, nullptr, nullptr, st)) return rc_;
    QES_LAUNCH_CHECK();
    return QES_OK;
  }
  return apply_ohu<T, V>(ns, nh, n_samples, bits, tt, eloc, L.wmean, 1.0 / (double)n_samples, L, 0.0, nullptr, F,
                         nullptr, st);
}

static int check_ws(int dtype, int ns, int nh, int64_t n_samples, void* ws, size_t ws_bytes, SRWork* L) {
  *L = sr_layout(dtype, ns, nh, n_samples, (char*)ws);
  if (!ws || ws_bytes < L->total) {
    qes_set_last_message("SR: workspace too small");
    return QES_ERR_WORKSPACE;
  }
  if (g_sr_impl.load() == 2 && !L->tc) {
    qes_set_last_message("SR: tensor-core path required but the shapes are outside its limits "
                         "(ns <= 127, nh <= 256, shared-memory budget)");
    return QES_ERR_SIZE;
  }
  return QES_OK;
}

extern "C" int qes_sr_tc_plan(int dtype, int ns, int nh, int64_t n_samples, int32_t* out, int n_out) {
  QES_ARG_CHECK(out && n_out > 0 && ns > 0 && nh > 0 && n_samples > 0, "qes_sr_tc_plan: bad args");
  QES_ARG_CHECK(dtype == QES_DTYPE_F32 || dtype == QES_DTYPE_C64, "qes_sr_tc_plan: bad dtype");
  const SRWork L = sr_layout(dtype, ns, nh, n_samples, nullptr);
  const TcDims& d = L.td;
  const int32_t f[19] = {L.tc ? 1 : 0, d.big ? 1 : 0, d.KC, d.n_chunks, d.nsplit, d.n_tiles, d.Kd, d.NB, d.Np,
                         d.MT, d.NC, d.NR, d.nnc, d.SPC, d.ov_stages, d.cl, d.sv ? 1 : 0, d.sv ? d.sv_grid : 0,
                         d.ovz ? 1 : 0};
  for (int k = 0; k < n_out; ++k) out[k] = k < 19 ? f[k] : 0;
  return QES_OK;
}

extern "C" int qes_sr_uses_tensor_cores(int dtype, int ns, int nh, int64_t n_samples, int* uses) {
  QES_ARG_CHECK(uses && ns > 0 && nh > 0 && n_samples > 0, "qes_sr_uses_tensor_cores: bad args");
  QES_ARG_CHECK(dtype == QES_DTYPE_F32 || dtype == QES_DTYPE_C64, "qes_sr_uses_tensor_cores: bad dtype");
  *uses = sr_layout(dtype, ns, nh, n_samples, nullptr).tc ? 1 : 0;
  return QES_OK;
}

static int sr_prepare(int dtype, int64_t n_samples, const uint32_t* bits, const void* tt, const SRWork& L,
                      cudaStream_t st);
static int sr_check_status(const SRWork& L, cudaStream_t st, bool cg_words = false);

extern "C" int qes_sr_force_weighted(int dtype, int ns, int nh, int64_t n_samples, const uint32_t* bits,
                                     const void* tanh_theta, const void* eloc, const float* probs, void* force_out,
                                     void* workspace, size_t workspace_bytes, void* stream) {
  QES_ARG_CHECK(ns > 0 && nh > 0 && n_samples > 0 && bits && tanh_theta && eloc && force_out, "qes_sr_force: bad args");
  QES_ARG_CHECK(dtype == QES_DTYPE_F32 || dtype == QES_DTYPE_C64, "qes_sr_force: bad dtype");
  SRWork L;
  int rc = check_ws(dtype, ns, nh, n_samples, workspace, workspace_bytes, &L);
  if (rc) return rc;
  L.wts = L.tw.wts = probs;
  cudaStream_t st = (cudaStream_t)stream;
  rc = sr_prepare(dtype, n_samples, bits, tanh_theta, L, st);
  if (rc) return rc;
  if (dtype == QES_DTYPE_F32)
    rc = sr_force_t<float>(ns, nh, n_samples, bits, (const float*)tanh_theta, (const float2*)eloc,
                           (double*)force_out, L, st);
  else
    rc = sr_force_t<float2>(ns, nh, n_samples, bits, (const float2*)tanh_theta, (const float2*)eloc,
                            (double2*)force_out, L, st);
  if (rc) return rc;
  return sr_check_status(L, st);
}

extern "C" int qes_sr_force(int dtype, int ns, int nh, int64_t n_samples, const uint32_t* bits,
                            const void* tanh_theta, const void* eloc, void* force_out, void* workspace,
                            size_t workspace_bytes, void* stream) {
  return qes_sr_force_weighted(dtype, ns, nh, n_samples, bits, tanh_theta, eloc, nullptr, force_out, workspace,
                               workspace_bytes, stream);
}

// grid-barrier test hook of the fused kernels (qes_sr_set_barrier_test)
static std::atomic<unsigned int> g_bar_extra{0};
static std::atomic<unsigned int> g_bar_limit{kGridBarLimit};

template <class T>
static int sr_matvec_t(int ns, int nh, int64_t n_samples, const uint32_t* bits, const T* tt, double shift,
                       const typename VecT<T>::type* v, typename VecT<T>::type* y, double* dot_part, const SRWork& L,
                       cudaStream_t st, bool vp_ready = false, const double* cg_done = nullptr,
                       const typename VecT<T>::type* pold = nullptr, const typename VecT<T>::type* sold = nullptr) {
  using V = typename VecT<T>::type;
  if (L.tc) {
    const int dtype = ScalarTraits<T>::is_complex ? QES_DTYPE_C64 : QES_DTYPE_F32;
    int rc = tc_matvec(dtype, L.td, n_samples, bits, tt, v, L.w, L.partial, L.tw, st, !vp_ready, cg_done,
                       BarCfg{g_bar_extra.load(), g_bar_limit.load()});
    if (rc) return rc;
    const int64_t P = (int64_t)ns + nh + (int64_t)ns * nh;
    const int pfr = qes_prof_begin(QES_PROF_REDUCE, st);
    if (int rc_ = launch_reduce_splits<T, V>(P, L.mv_nsplit, L.partial, shift, v, y,
        dot_part, dot_part ? L.scal : nullptr, L.counter, st, cg_done, pold, sold)) return rc_;
    QES_LAUNCH_CHECK();
    qes_prof_end(pfr, st);
    return QES_OK;
  }
  int rc = apply_ov<T, V>(ns, nh, n_samples, bits, tt, v, L.w, L.wmean, L, st, cg_done);
  if (rc) return rc;
  return apply_ohu<T, V>(ns, nh, n_samples, bits, tt, L.w, L.wmean, 1.0 / (double)n_samples, L, shift, v, y,
                         dot_part, st, cg_done, pold, sold);
}

// per-step operands of the tensor-core path (spins as BF16 tiles) and the status word
static int sr_prepare(int dtype, int64_t n_samples, const uint32_t* bits, const void* tt, const SRWork& L,
                      cudaStream_t st) {
  if (!L.tc) return QES_OK;
  return tc_prepare_step(dtype, L.td, n_samples, bits, tt, L.tw, st);
}

// Reads the tensor-core status word and, inside a CG solve (cg_words: counter[4] was zeroed at the
// start of the solve), the grid-barrier error word of the fused CG kernel; synchronises the stream.
static int sr_check_status(const SRWork& L, cudaStream_t st, bool cg_words) {
  int h[2] = {0, 0};
  if (L.tc) QES_CUDA_CHECK(cudaMemcpyAsync(&h[0], L.tw.status, sizeof(int), cudaMemcpyDeviceToHost, st));
  if (cg_words) QES_CUDA_CHECK(cudaMemcpyAsync(&h[1], L.counter + 4, sizeof(int), cudaMemcpyDeviceToHost, st));
  QES_CUDA_CHECK(cudaStreamSynchronize(st));
  if (h[0] != 0) {
    qes_set_last_message("SR tensor-core matvec: a bounded device wait gave up");
    return QES_ERR_TIMEOUT;
  }
  if (h[1] != 0) {
    qes_set_last_message("SR CG: a bounded grid-barrier wait gave up");
    return QES_ERR_TIMEOUT;
  }
  return QES_OK;
}

extern "C" int qes_sr_matvec_weighted(int dtype, int ns, int nh, int64_t n_samples, const uint32_t* bits,
                                      const void* tanh_theta, const float* probs, double shift, const void* v,
                                      void* y_out, void* workspace, size_t workspace_bytes, void* stream) {
  QES_ARG_CHECK(ns > 0 && nh > 0 && n_samples > 0 && bits && tanh_theta && v && y_out, "qes_sr_matvec: bad args");
  QES_ARG_CHECK(dtype == QES_DTYPE_F32 || dtype == QES_DTYPE_C64, "qes_sr_matvec: bad dtype");
  SRWork L;
  int rc = check_ws(dtype, ns, nh, n_samples, workspace, workspace_bytes, &L);
  if (rc) return rc;
  L.wts = L.tw.wts = probs;
  cudaStream_t st = (cudaStream_t)stream;
  rc = sr_prepare(dtype, n_samples, bits, tanh_theta, L, st);
  if (rc) return rc;
  if (dtype == QES_DTYPE_F32)
    rc = sr_matvec_t<float>(ns, nh, n_samples, bits, (const float*)tanh_theta, shift, (const double*)v,
                            (double*)y_out, nullptr, L, st);
  else
    rc = sr_matvec_t<float2>(ns, nh, n_samples, bits, (const float2*)tanh_theta, shift, (const double2*)v,
                             (double2*)y_out, nullptr, L, st);
  if (rc) return rc;
  return sr_check_status(L, st);
}

extern "C" int qes_sr_matvec(int dtype, int ns, int nh, int64_t n_samples, const uint32_t* bits,
                             const void* tanh_theta, double shift, const void* v, void* y_out, void* workspace,
                             size_t workspace_bytes, void* stream) {
  return qes_sr_matvec_weighted(dtype, ns, nh, n_samples, bits, tanh_theta, nullptr, shift, v, y_out, workspace,
                                workspace_bytes, stream);
}

// ----------------------------------------------------------------------------
// CUDA graph of one chunk of CG iterations (matvec + x/r update + direction
// update, `check_every` times), captured on a private stream and replayed
// while the kernel arguments stay the same (same buffers, sizes and shift).
// ----------------------------------------------------------------------------
#include <mutex>
#include <cstring>

namespace {
struct CgGraphKey {
  const void* bits; const void* tt; const void* ws; const void* wts; int64_t n; int ns, nh, dtype, chunk, tc, l2;
  int big, kc, nsplit, nnc, nc, spc, cl;  // tiling of the captured kernels
  int bartest;                             // grid-barrier test hook armed (also keeps the struct free of padding)
  double shift;
  bool operator==(const CgGraphKey& o) const { return std::memcmp(this, &o, sizeof(*this)) == 0; }
};
static_assert(sizeof(CgGraphKey) == 4 * sizeof(void*) + 8 + 14 * 4 + 8, "CgGraphKey has padding bytes (memcmp key)");
struct CgGraphSlot {
  bool init = false;
  cudaStream_t cs = nullptr;
  cudaEvent_t ev_in = nullptr, ev_out = nullptr;
  cudaGraphExec_t exec = nullptr;
  CgGraphKey key{};
  long long nodes = 0;
  // device loop: a counter reset, then a WHILE node whose body is one chunk + the loop condition
  cudaGraphExec_t lexec = nullptr;
  CgGraphKey lkey{};
  unsigned lmax = 0;
  long long lnodes = 0;            // launches of one body (the chunk and the condition kernel)
  bool lfailed = false;            // this key could not be built as a device loop: host-driven chunks
};
constexpr int kMaxGraphDevices = 64;
std::mutex g_graph_mu;
CgGraphSlot g_graph[kMaxGraphDevices];
std::atomic<int> g_use_graphs{1};
std::atomic<int> g_l2_persist{0};
std::atomic<int> g_cg_fused{1};            // automatic
std::atomic<int> g_cg_loop{1};             // device-side loop over the CG chunks

// L2 persistence of the tensor-core operands across the CG iterations: an access-policy window
// over the BF16 tiles (T rows, T^T, Sigma^T, V') on the launching stream, sized to the device's
// persisting-L2 limit; cleared (and the persisting lines released) after the solve.
struct L2Props { bool init = false; size_t max_persist = 0, max_window = 0; };
L2Props g_l2_props[kMaxGraphDevices];

void l2_window(cudaStream_t st, int dev, const void* base, size_t bytes) {
  if (dev < 0 || dev >= kMaxGraphDevices) return;
  L2Props& pr = g_l2_props[dev];
  if (!pr.init) {
    int v = 0;
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMaxPersistingL2CacheSize, dev) == cudaSuccess) pr.max_persist = (size_t)v;
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMaxAccessPolicyWindowSize, dev) == cudaSuccess) pr.max_window = (size_t)v;
    pr.init = true;
  }
  if (pr.max_persist == 0 || pr.max_window == 0) return;
  cudaStreamAttrValue a;
  std::memset(&a, 0, sizeof(a));
  if (bytes > 0) {
    const size_t nb = std::min(bytes, pr.max_window);
    const size_t lim = std::min(nb, pr.max_persist);
    cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, lim);
    a.accessPolicyWindow.base_ptr = const_cast<void*>(base);
    a.accessPolicyWindow.num_bytes = nb;
    a.accessPolicyWindow.hitRatio = (float)std::min(1.0, (double)lim / (double)nb);
    a.accessPolicyWindow.hitProp = cudaAccessPropertyPersisting;
    a.accessPolicyWindow.missProp = cudaAccessPropertyStreaming;
  }
  cudaStreamSetAttribute(st, cudaStreamAttributeAccessPolicyWindow, &a);
  if (bytes == 0) cudaCtxResetPersistingL2Cache();
  cudaGetLastError();           // an unsupported policy leaves the solve unaffected
}
}  // namespace

// The loop condition of the device-driven CG: one more chunk while the solve has not converged,
// no bounded wait has given up, and fewer than max_chunks chunks have run.  The counter makes the
// loop finite whatever the other kernels do.
// entry of the device loop: no chunk when the solve has already converged (or a wait gave up)
__global__ void cg_loop_reset_kernel(unsigned int* count, cudaGraphConditionalHandle h, const double* __restrict__ scal,
                                     const int* __restrict__ status, const int* __restrict__ bar_err) {
  *count = 0u;
  const bool run = scal[4] == 0.0 && (status == nullptr || *status == 0) && *bar_err == 0;
  cudaGraphSetConditional(h, run ? 1u : 0u);
}
__global__ void cg_loop_cond_kernel(cudaGraphConditionalHandle h, const double* __restrict__ scal,
                                    unsigned int* __restrict__ count, unsigned int max_chunks,
                                    const int* __restrict__ status, const int* __restrict__ bar_err) {
  const unsigned int c = *count + 1u;
  *count = c;
  const bool more = scal[4] == 0.0 && c < max_chunks && (status == nullptr || *status == 0) && *bar_err == 0;
  cudaGraphSetConditional(h, more ? 1u : 0u);
}

extern "C" int qes_set_cg_device_loop(int enable) {
  g_cg_loop.store(enable ? 1 : 0);
  return QES_OK;
}

extern "C" int qes_sr_set_barrier_test(unsigned int extra_arrivals, unsigned int poll_limit) {
  if (extra_arrivals > 1u || (extra_arrivals == 0u) != (poll_limit == 0u)) {
    qes_set_last_message("qes_sr_set_barrier_test: (0, 0) restores normal barriers; (1, polls) arms the test");
    return QES_ERR_ARG;
  }
  g_bar_extra.store(extra_arrivals);
  g_bar_limit.store(extra_arrivals ? std::min(poll_limit, kGridBarLimit) : kGridBarLimit);
  return QES_OK;
}

// the fused cooperative vector kernel launched by programmatic dependent launch instead of as a
// cooperative launch (its prologue then overlaps the O^H u kernel's tail): on by default (TFIM-16 CG
// iteration 18.8 -> 18.3 us, 6x6 J1-J2 and the forced 10x10 form within 0.3 us; bit-identical)
static std::atomic<int> g_cg_fused_pdl{1};
extern "C" int qes_set_cg_fused_pdl(int on) {
  g_cg_fused_pdl.store(on ? 1 : 0);
  return QES_OK;
}
// x/r and direction updates of the standard CG step in one launch with a grid barrier
// (cg_xrp_kernel): on by default
static std::atomic<int> g_cg_xrp{1};
extern "C" int qes_set_cg_xrp(int on) {
  g_cg_xrp.store(on ? 1 : 0);
  return QES_OK;
}
// Chronopoulos-Gear CG steps (the matvec of r, one reduction, one update kernel) on the kernel-chain
// path: off by default -- one kernel and one grid-wide reduction fewer per step (heis10x10 CG
// iteration 43.3 -> 40.3 us, the same 136 iterations), but the s = A p recurrence does not damp the
// rounding of a float32 / BF16-split operator, and on strongly rank-deficient systems (20x20 TFIM,
// 256 samples, P = 642,000, shift 1e-4) it failed to converge within 3,000 steps where the
// standard form converges
static std::atomic<int> g_cg_single{0};
extern "C" int qes_set_cg_single_reduction(int on) {
  g_cg_single.store(on ? 1 : 0);
  return QES_OK;
}
extern "C" int qes_set_cg_fused(int mode) {
  if (mode < 0 || mode > 3) {
    qes_set_last_message("qes_set_cg_fused: mode 0 (off), 1 (automatic), 2 (always) or 3 (always, one CTA per SM)");
    return QES_ERR_ARG;
  }
  g_cg_fused.store(mode);
  return QES_OK;
}

extern "C" int qes_set_l2_persist(int enable) {
  g_l2_persist.store(enable ? 1 : 0);
  return QES_OK;
}

extern long long qes_launch_count(int reset);
void qes_count_launches(int n);

extern "C" int qes_set_cg_graphs(int enable) {
  g_use_graphs.store(enable ? 1 : 0);
  return QES_OK;
}

// Jacobi preconditioner D^-1 = 1 / diag(S + shift) into L.dinv: Obar^H = O^H p / Ns by the O^H pass
// (g = 1, no centring; into L.Ap, free before the iterations), the weighted column means of |t|^2,
// then diag(S)_k = mean|O_k|^2 - |Obar_k|^2 (clamped at 0)
template <class T>
static int sr_jacobi_t(int ns, int nh, int64_t n_samples, const uint32_t* bits, const T* tt, double shift,
                       const SRWork& L, cudaStream_t st) {
  using V = typename VecT<T>::type;
  const int64_t P = (int64_t)ns + nh + (int64_t)ns * nh;
  float2* ones = (float2*)L.wpart;                       // scratch of at least Ns float2
  fill_ones_kernel<<<RED_BLOCKS, RED_THREADS, 0, st>>>(n_samples, ones);
  QES_LAUNCH_CHECK();
  V* obar_h = (V*)L.Ap;
  const double inv_n = 1.0 / (double)n_samples;
  if (L.tc) {
    const int dtype = ScalarTraits<T>::is_complex ? QES_DTYPE_C64 : QES_DTYPE_F32;
    int rc = tc_ohu(dtype, L.td, n_samples, ones, nullptr, 0, inv_n, L.partial, L.tw, st);
    if (rc) return rc;
    if ((rc = launch_reduce_splits<T, V>(P, L.nsplit, L.partial, 0.0, nullptr, obar_h, nullptr, nullptr, nullptr,
                                         st)))
      return rc;
    QES_LAUNCH_CHECK();
  } else if (int rc = apply_ohu<T, V>(ns, nh, n_samples, bits, tt, ones, nullptr, inv_n, L, 0.0, nullptr, obar_h,
                                      nullptr, st)) {
    return rc;
  }
  double* part = L.tsq + nh;
  tsq_part_kernel<T><<<dim3((nh + 31) / 32, TSQ_SPLITS), dim3(32, 8), 0, st>>>(nh, n_samples, tt, L.wts, part);
  tsq_sum_kernel<<<(nh + 255) / 256, 256, 0, st>>>(nh, TSQ_SPLITS, inv_n, part, L.tsq);
  jacobi_dinv_kernel<V><<<RED_BLOCKS, RED_THREADS, 0, st>>>(ns, nh, P, L.tsq, obar_h, shift, L.dinv);
  QES_LAUNCH_CHECK_N(3);
  return QES_OK;
}

// x0: start of the iteration for the unscaled system (nullptr: zero)
template <class T>
static int sr_cg_t(int ns, int nh, int64_t n_samples, const uint32_t* bits, const T* tt, const float2* eloc,
                   const qes_sr_options* opt, typename VecT<T>::type* x_out, qes_sr_result* res, const SRWork& L,
                   cudaStream_t st, const typename VecT<T>::type* x0 = nullptr) {
  using V = typename VecT<T>::type;
  const int64_t P = (int64_t)ns + nh + (int64_t)ns * nh;
  V* x = (V*)L.x; V* r = (V*)L.r; V* p = (V*)L.p; V* Ap = (V*)L.Ap; V* b = (V*)L.b;
  const int dtype = ScalarTraits<T>::is_complex ? QES_DTYPE_C64 : QES_DTYPE_F32;
  int rc = sr_prepare(dtype, n_samples, bits, tt, L, st);
  if (rc) return rc;
  // b = F
  rc = sr_force_t<T>(ns, nh, n_samples, bits, tt, eloc, b, L, st);
  if (rc) return rc;
  // the energy mean stays on the device (scal[12..13]) until the final read of the solver state
  QES_CUDA_CHECK(cudaMemcpyAsync(L.scal + 12, L.wmean, 2 * sizeof(double), cudaMemcpyDeviceToDevice, st));
  QES_CUDA_CHECK(cudaMemsetAsync(L.counter, 0, 128 * sizeof(unsigned int), st));
  // preconditioned CG (SciPy's cg with M = D^-1): z = D^-1 r in the direction update, rho = r^H z
  const double* dinv = nullptr;
  if (opt->precond == QES_PRECOND_JACOBI) {
    rc = sr_jacobi_t<T>(ns, nh, n_samples, bits, tt, opt->shift, L, st);
    if (rc) return rc;
    dinv = L.dinv;
  }
  double* parts_z = dinv ? L.parts + 2 * RED_BLOCKS : nullptr;
  if (x0) {
    // warm start: x = x0, r = b - (S + shift) x0, p = D^-1 r; the threshold stays rtol * ||b||
    QES_CUDA_CHECK(cudaMemcpyAsync(x, x0, P * sizeof(V), cudaMemcpyDeviceToDevice, st));
    rc = sr_matvec_t<T>(ns, nh, n_samples, bits, tt, opt->shift, x, Ap, nullptr, L, st, false);
    if (rc) return rc;
    cg_init_x0_kernel<V><<<RED_BLOCKS, RED_THREADS, 0, st>>>(P, b, Ap, r, p, dinv);
    norm2_kernel<V><<<RED_BLOCKS, RED_THREADS, 0, st>>>(P, b, L.parts);
    norm2_kernel<V><<<RED_BLOCKS, RED_THREADS, 0, st>>>(P, r, L.parts + RED_BLOCKS);
    QES_LAUNCH_CHECK_N(3);
    if (dinv) {
      wnorm2_kernel<V><<<RED_BLOCKS, RED_THREADS, 0, st>>>(P, r, dinv, parts_z);
      QES_LAUNCH_CHECK();
    }
    cg_setup_kernel<<<1, SC_THREADS, 0, st>>>(RED_BLOCKS, L.parts, opt->rtol, opt->atol, L.scal, L.parts + RED_BLOCKS,
                                              parts_z);
    QES_LAUNCH_CHECK();
  } else {
    cg_init_kernel<V><<<RED_BLOCKS, RED_THREADS, 0, st>>>(P, b, x, r, p, dinv);
    norm2_kernel<V><<<RED_BLOCKS, RED_THREADS, 0, st>>>(P, b, L.parts);
    QES_LAUNCH_CHECK_N(2);
    if (dinv) {
      wnorm2_kernel<V><<<RED_BLOCKS, RED_THREADS, 0, st>>>(P, b, dinv, parts_z);
      QES_LAUNCH_CHECK();
    }
    cg_setup_kernel<<<1, SC_THREADS, 0, st>>>(RED_BLOCKS, L.parts, opt->rtol, opt->atol, L.scal, nullptr, parts_z);
    QES_LAUNCH_CHECK();
  }
  const int check = opt->check_every > 0 ? opt->check_every : 8;
  // No host read before the first chunk: a system that needs no iteration (||F|| <= atol) has its
  // converged flag set by cg_setup_kernel, and every CG kernel then returns at once.
  double hs[16] = {0};
  int it = 0;
  bool done = false;
  // fused vector kernel (split reduction, x/r and direction updates with two grid barriers):
  // always (2), never (0), or automatically (1) for grids of up to 160 CTAs
  const int fused_mode = g_cg_fused.load();
  bool fused = fused_mode != 0 && !L.fp64;         // the fused kernel reads float32 split partials
  int fused_grid = 0, fused_cv = 1;
  constexpr int FEV = (int)(16 / sizeof(T));
  const bool fused_vec = (P % FEV == 0) && ((reinterpret_cast<uintptr_t>(L.partial) & 15) == 0);
  if (fused) {
    int dv_ = 0, nsm = 0, per_sm = 0;
    QES_CUDA_CHECK(cudaGetDevice(&dv_));
    QES_CUDA_CHECK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dv_));
    if (fused_vec)
      QES_CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, cg_fused_kernel<T, V, true>,
                                                                   CF_TX * CF_TY, 0));
    else
      QES_CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, cg_fused_kernel<T, V, false>,
                                                                   CF_TX * CF_TY, 0));
    // column vectors per block pass as in the standalone split reduction, the grid within residency
    // mode 3: one CTA per SM (the grid barriers then wait for fewer arrivals)
    const int64_t cap = std::min<int64_t>((int64_t)nsm * (fused_mode == 3 ? 1 : std::max(per_sm, 1)), RED_BLOCKS);
    const int64_t nvec = fused_vec ? P / FEV : P;
    int64_t cv = (nvec + cap - 1) / cap;
    const int nthr = CF_TX * CF_TY;
    cv = std::max<int64_t>(cv, nthr / std::max(L.mv_nsplit, 1));
    const int64_t need = (L.mv_nsplit + RS_BATCH - 1) / RS_BATCH;
    cv = std::min<int64_t>(cv, std::max<int64_t>(nthr / std::max<int64_t>(need, 1), 1));
    cv = std::max<int64_t>(1, std::min<int64_t>(cv, 128));
    fused_cv = (int)cv;
    fused_grid = (int)std::max<int64_t>(1, std::min<int64_t>(cap, (nvec + cv - 1) / cv));
    // automatic: up to 160 CTAs (measured per CG iteration, fused vs three kernels: TFIM-16 19.9 vs
    // 22.7 us, 6x6 J1-J2 (158 CTAs) 44.6 vs 45.7 us, 10x10 Heisenberg (290 CTAs) 46.3 vs 45.5 us)
    if (fused_mode == 1 && fused_grid > 160) fused = false;
  }
  const BarCfg bcfg{g_bar_extra.load(), g_bar_limit.load()};
  const bool single = !fused && dinv == nullptr && g_cg_single.load() != 0;
  const bool xrp = !fused && !single && g_cg_xrp.load() != 0;
  auto run_direct = [&](int nrun, int it0) -> int {
    for (int q = 0; q < nrun; ++q) {
      if (fused) {
        // O v and O^H u (split partials), then the fused vector kernel
        if (L.tc) {
          const int dtype_ = ScalarTraits<T>::is_complex ? QES_DTYPE_C64 : QES_DTYPE_F32;
          int r2 = tc_matvec(dtype_, L.td, n_samples, bits, tt, p, L.w, L.partial, L.tw, st, it0 + q == 0,
                             L.scal + 4, bcfg);
          if (r2) return r2;
        } else {
          int r2 = apply_ov<T, V>(ns, nh, n_samples, bits, tt, p, L.w, L.wmean, L, st, L.scal + 4);
          if (r2) return r2;
          r2 = launch_ohu_plain<T>(ns, nh, n_samples, bits, tt, L.w, L.wmean, 1.0 / (double)n_samples,
                                   L.partial, st, L.scal + 4, L.wts);
          if (r2) return r2;
        }
        cudaLaunchConfig_t lc = {};
        lc.gridDim = dim3(fused_grid);
        lc.blockDim = dim3(CF_TX, CF_TY);
        lc.dynamicSmemBytes = 0;
        lc.stream = st;
        cudaLaunchAttribute at[1];
        if (g_cg_fused_pdl.load() != 0 && qes_pdl_on()) {
          at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
          at[0].val.programmaticStreamSerializationAllowed = 1;
        } else {
          at[0].id = cudaLaunchAttributeCooperative;
          at[0].val.cooperative = 1;
        }
        lc.attrs = at;
        lc.numAttrs = 1;
        const int pfr = qes_prof_begin(QES_PROF_REDUCE, st);
        if (fused_vec)
          QES_CUDA_CHECK(cudaLaunchKernelEx(&lc, cg_fused_kernel<T, V, true>, P, L.mv_nsplit, fused_cv,
                                            (const T*)L.partial, opt->shift, x, r, p, Ap, L.scal, L.parts,
                                            L.counter + 32, (int*)(L.counter + 4), L.td,
                                            L.tc ? L.tw.vp : (uint16_t*)nullptr, bcfg, dinv));
        else
          QES_CUDA_CHECK(cudaLaunchKernelEx(&lc, cg_fused_kernel<T, V, false>, P, L.mv_nsplit, fused_cv,
                                            (const T*)L.partial, opt->shift, x, r, p, Ap, L.scal, L.parts,
                                            L.counter + 32, (int*)(L.counter + 4), L.td,
                                            L.tc ? L.tw.vp : (uint16_t*)nullptr, bcfg, dinv));
        qes_prof_end(pfr, st);
        QES_LAUNCH_CHECK();
        continue;
      }
      if (single) {
        // Chronopoulos-Gear step: the matvec of r, one reduction (r^H A r, |r|^2, alpha, beta,
        // the convergence test), one update kernel
        int r2 = sr_matvec_t<T>(ns, nh, n_samples, bits, tt, opt->shift, r, Ap, L.parts, L, st,
                                /*vp_ready=*/it0 + q > 0, L.scal + 4, (const V*)p, (const V*)L.mw1);
        if (r2) return r2;
        QES_CUDA_CHECK(qes_launch_pdl(cg_cgstep_kernel<V>, dim3(vec_blocks(P)), dim3(RED_THREADS), 0, st, P,
                                      (const V*)Ap, x, r, p, (V*)L.mw1, (const double*)L.scal, L.td,
                                      L.tc ? L.tw.vp : (uint16_t*)nullptr));
        QES_LAUNCH_CHECK();
        continue;
      }
      int r2 = sr_matvec_t<T>(ns, nh, n_samples, bits, tt, opt->shift, p, Ap, L.parts, L, st,
                              /*vp_ready=*/it0 + q > 0, L.scal + 4);
      if (r2) return r2;
      // (alpha is computed by the last block of the matvec's split reduction)
      if (xrp) {
        QES_CUDA_CHECK(qes_launch_pdl(cg_xrp_kernel<V>, dim3(vec_blocks(P)), dim3(RED_THREADS), 0, st, P,
                                      (const V*)Ap, x, r, p, L.scal, L.parts, L.counter + 32, (int*)(L.counter + 4),
                                      L.td, L.tc ? L.tw.vp : (uint16_t*)nullptr, bcfg, dinv));
        QES_LAUNCH_CHECK();
        continue;
      }
      QES_CUDA_CHECK(qes_launch_pdl(cg_xr_kernel<V>, dim3(vec_blocks(P)), dim3(RED_THREADS), 0, st, P, (const V*)p,
                                    (const V*)Ap, x, r, L.scal, L.parts, L.counter + 1, dinv,
                                    dinv ? L.parts + RED_BLOCKS : (double*)nullptr));
      QES_CUDA_CHECK(qes_launch_pdl(cg_p_kernel<V>, dim3(vec_blocks(P)), dim3(RED_THREADS), 0, st, P, (const V*)r, p,
                                    (const double*)L.scal, L.td, L.tc ? L.tw.vp : (uint16_t*)nullptr, dinv));
      QES_LAUNCH_CHECK_N(2);
    }
    return QES_OK;
  };
  int dev = 0;
  QES_CUDA_CHECK(cudaGetDevice(&dev));
  const bool graphs = g_use_graphs.load() != 0 && !qes_prof_on() && dev >= 0 && dev < kMaxGraphDevices;
  const bool l2 = L.tc && g_l2_persist.load() != 0;
  const size_t l2_bytes = l2 ? (size_t)((const char*)L.tw.wsum - (const char*)L.tw.t_rows) : 0;
  if (l2) {
    l2_window(st, dev, L.tw.t_rows, l2_bytes);
    if (graphs && g_graph[dev].init) l2_window(g_graph[dev].cs, dev, L.tw.t_rows, l2_bytes);
  }
  while (!done && it < opt->maxiter) {
    const int nrun = std::min(check, opt->maxiter - it);
    // set when the device loop was launched: its chunk count is read back after the lock is released
    unsigned int* loop_count = nullptr;
    unsigned loop_max = 0;
    long long loop_nodes = 0;
    if (!graphs || it == 0 || nrun != check) {
      rc = run_direct(nrun, it);
      if (rc) return rc;
      // the first chunk goes on to the device loop without a host read: the loop checks the
      // converged flag before its first chunk
      if (it == 0 && graphs && g_cg_loop.load() != 0 && nrun == check && (opt->maxiter - nrun) / check >= 2) {
        it += nrun;
        continue;
      }
    } else {
      std::lock_guard<std::mutex> lock(g_graph_mu);
      CgGraphSlot& gs = g_graph[dev];
      if (!gs.init) {
        QES_CUDA_CHECK(cudaStreamCreateWithFlags(&gs.cs, cudaStreamNonBlocking));
        QES_CUDA_CHECK(cudaEventCreateWithFlags(&gs.ev_in, cudaEventDisableTiming));
        QES_CUDA_CHECK(cudaEventCreateWithFlags(&gs.ev_out, cudaEventDisableTiming));
        gs.init = true;
        if (l2) l2_window(gs.cs, dev, L.tw.t_rows, l2_bytes);
      }
      const CgGraphKey key{bits, tt, L.w, L.wts, n_samples, ns, nh, ScalarTraits<T>::is_complex ? 1 : 0, nrun,
                           L.tc ? 1 : 0, (l2 ? 1 : 0) | (fused ? 2 : 0) | (dinv ? 4 : 0), L.td.big ? 1 : 0,
                           L.td.KC, L.mv_nsplit,
                           L.td.nnc, L.td.NC, L.td.SPC,
                           L.td.cl | (L.td.sv ? 4 : 0) | (L.td.ovz ? 8 : 0) | (L.td.splitc ? 16 : 0) | (single ? 32 : 0) |
                               (xrp ? 64 : 0) | (L.td.prefetch ? 128 : 0) | (g_cg_fused_pdl.load() ? 256 : 0),
                           (int)bcfg.extra, opt->shift};
      if (gs.exec == nullptr || !(gs.key == key)) {
        if (gs.exec) {
          cudaGraphExecDestroy(gs.exec);
          gs.exec = nullptr;
        }
        const long long before = qes_launch_count(0);
        QES_CUDA_CHECK(cudaStreamBeginCapture(gs.cs, cudaStreamCaptureModeThreadLocal));
        cudaStream_t saved = st;
        st = gs.cs;
        const int rcap = run_direct(nrun, 1);
        st = saved;
        cudaGraph_t g = nullptr;
        const cudaError_t ec = cudaStreamEndCapture(gs.cs, &g);
        if (rcap) return rcap;
        if (ec != cudaSuccess) { qes_set_last_error(ec, "cudaStreamEndCapture"); return QES_ERR_CUDA; }
        const cudaError_t ei = cudaGraphInstantiate(&gs.exec, g, 0);
        cudaGraphDestroy(g);
        if (ei != cudaSuccess) { gs.exec = nullptr; qes_set_last_error(ei, "cudaGraphInstantiate"); return QES_ERR_CUDA; }
        gs.nodes = qes_launch_count(0) - before;
        qes_count_launches((int)-gs.nodes);     // captured, not run
        gs.key = key;
      }
      // Device loop: the remaining full chunks in one launch of a graph whose WHILE node repeats
      // the chunk until the converged flag is set (no host round trip per chunk).  Built once per
      // key; where the driver rejects it, the chunks stay host-driven.
      const unsigned lmax = (unsigned)((opt->maxiter - it) / check);
      unsigned int* lcount = L.counter + 96;  // own 128-byte line
      if (g_cg_loop.load() != 0 && lmax >= 2 &&
          !(gs.lfailed && gs.lkey == key && gs.lmax == lmax)) {
        if (gs.lexec == nullptr || !(gs.lkey == key) || gs.lmax != lmax) {
          if (gs.lexec) {
            cudaGraphExecDestroy(gs.lexec);
            gs.lexec = nullptr;
          }
          gs.lkey = key;
          gs.lmax = lmax;
          gs.lfailed = true;                  // until the build below succeeds
          cudaGraph_t g = nullptr;
          bool ok = cudaGraphCreate(&g, 0) == cudaSuccess;
          cudaGraphNode_t n0 = nullptr, n1 = nullptr;
          cudaGraphConditionalHandle hnd = 0;
          if (ok) ok = cudaGraphConditionalHandleCreate(&hnd, g, 0u, cudaGraphCondAssignDefault) == cudaSuccess;
          if (ok) {
            const double* scal_arg = L.scal;
            const int* status_arg = L.tc ? L.tw.status : nullptr;
            const int* barerr_arg = (const int*)(L.counter + 4);
            void* kargs[] = {(void*)&lcount, (void*)&hnd, (void*)&scal_arg, (void*)&status_arg, (void*)&barerr_arg};
            cudaKernelNodeParams kp = {};
            kp.func = (void*)cg_loop_reset_kernel;
            kp.gridDim = dim3(1);
            kp.blockDim = dim3(1);
            kp.kernelParams = kargs;
            ok = cudaGraphAddKernelNode(&n0, g, nullptr, 0, &kp) == cudaSuccess;
          }
          cudaGraph_t body = nullptr;
          if (ok) {
            cudaGraphNodeParams cp = {};
            cp.type = cudaGraphNodeTypeConditional;
            cp.conditional.handle = hnd;
            cp.conditional.type = cudaGraphCondTypeWhile;
            cp.conditional.size = 1;
            ok = cudaGraphAddNode(&n1, g, &n0, 1, &cp) == cudaSuccess;
            if (ok) body = cp.conditional.phGraph_out[0];
          }
          long long bnodes = 0;
          if (ok) {
            const long long before = qes_launch_count(0);
            ok = cudaStreamBeginCaptureToGraph(gs.cs, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal) ==
                 cudaSuccess;
            if (ok) {
              cudaStream_t saved = st;
              st = gs.cs;
              int rcap = run_direct(check, 1);
              if (!rcap) {
                cg_loop_cond_kernel<<<1, 1, 0, gs.cs>>>(hnd, L.scal, lcount, lmax, L.tc ? L.tw.status : nullptr,
                                                         (const int*)(L.counter + 4));
                if (cudaPeekAtLastError() != cudaSuccess) rcap = QES_ERR_CUDA;
                else qes_count_launches(1);
              }
              st = saved;
              cudaGraph_t bout = nullptr;
              const cudaError_t ec = cudaStreamEndCapture(gs.cs, &bout);
              ok = rcap == QES_OK && ec == cudaSuccess;
            }
            bnodes = qes_launch_count(0) - before;
            qes_count_launches((int)-bnodes);   // captured, not run
          }
          if (ok) ok = cudaGraphInstantiate(&gs.lexec, g, 0) == cudaSuccess;
          if (!ok) gs.lexec = nullptr;
          if (g) cudaGraphDestroy(g);
          cudaGetLastError();                   // a rejected build leaves no error behind
          if (ok) {
            gs.lfailed = false;
            gs.lnodes = bnodes;
          }
        }
        if (gs.lexec) {
          QES_CUDA_CHECK(cudaEventRecord(gs.ev_in, st));
          QES_CUDA_CHECK(cudaStreamWaitEvent(gs.cs, gs.ev_in, 0));
          if (cudaGraphLaunch(gs.lexec, gs.cs) != cudaSuccess) {
            cudaGetLastError();                 // rejected at launch: host-driven chunks from now on
            cudaGraphExecDestroy(gs.lexec);
            gs.lexec = nullptr;
            gs.lfailed = true;
          }
        }
        if (gs.lexec) {
          QES_CUDA_CHECK(cudaEventRecord(gs.ev_out, gs.cs));
          QES_CUDA_CHECK(cudaStreamWaitEvent(st, gs.ev_out, 0));
          loop_count = lcount;
          loop_max = lmax;
          loop_nodes = gs.lnodes;
        }
      }
      if (!loop_count) {
        QES_CUDA_CHECK(cudaEventRecord(gs.ev_in, st));
        QES_CUDA_CHECK(cudaStreamWaitEvent(gs.cs, gs.ev_in, 0));
        QES_CUDA_CHECK(cudaGraphLaunch(gs.exec, gs.cs));
        QES_CUDA_CHECK(cudaEventRecord(gs.ev_out, gs.cs));
        QES_CUDA_CHECK(cudaStreamWaitEvent(st, gs.ev_out, 0));
        qes_count_launches((int)gs.nodes);
      }
    }
    if (loop_count) {
      unsigned int chunks = 0;
      QES_CUDA_CHECK(cudaMemcpyAsync(&chunks, loop_count, sizeof(unsigned int), cudaMemcpyDeviceToHost, st));
      QES_CUDA_CHECK(cudaMemcpyAsync(hs, L.scal, 16 * sizeof(double), cudaMemcpyDeviceToHost, st));
      rc = sr_check_status(L, st, true);            // synchronises the stream
      if (rc) return rc;
      if (chunks > loop_max) {
        qes_set_last_message("SR CG: the device loop ran an impossible number of chunks");
        return QES_ERR_CUDA;
      }
      qes_count_launches((int)(1 + (long long)chunks * loop_nodes));
      it += (int)chunks * check;
      done = hs[4] != 0.0;
      continue;
    }
    it += nrun;
    QES_CUDA_CHECK(cudaMemcpyAsync(hs, L.scal, 16 * sizeof(double), cudaMemcpyDeviceToHost, st));
    rc = sr_check_status(L, st, true);          // synchronises the stream
    if (rc) return rc;
    done = hs[4] != 0.0;
  }
  if (l2) {
    l2_window(st, dev, nullptr, 0);
    if (graphs && g_graph[dev].init) l2_window(g_graph[dev].cs, dev, nullptr, 0);
  }
  // Chronopoulos-Gear steps test |r|^2 at the start of the next step: the residual of the last
  // step before maxiter is tested here (|r|^2 into scal[2]; r does not change after convergence)
  if (single) {
    norm2_kernel<V><<<RED_BLOCKS, RED_THREADS, 0, st>>>(P, r, L.parts);
    sum_parts_kernel<<<1, SC_THREADS, 0, st>>>(RED_BLOCKS, L.parts, L.scal + 2);
    QES_LAUNCH_CHECK_N(2);
  }
  // the final solver state (also when CG ran no chunk); a bounded wait of the force pass must
  // surface even when CG needed no iteration
  QES_CUDA_CHECK(cudaMemcpyAsync(hs, L.scal, 16 * sizeof(double), cudaMemcpyDeviceToHost, st));
  if ((rc = sr_check_status(L, st, true))) return rc;
  done = hs[4] != 0.0 || (single && hs[2] <= hs[3]);
  // true residual of the solution, ||F - (S + shift) x|| / ||F||, with one more matvec: CG's recursive
  // residual drifts from it once the rounding of the float32 / BF16-split contractions dominates
  double true_rr = -1.0;
  if (opt->maxiter > 0 && !opt->skip_true_residual) {
    rc = sr_matvec_t<T>(ns, nh, n_samples, bits, tt, opt->shift, x, Ap, nullptr, L, st, false);
    if (rc) return rc;
    diff_norm2_kernel<V><<<RED_BLOCKS, RED_THREADS, 0, st>>>(P, b, Ap, L.parts);
    sum_parts_kernel<<<1, SC_THREADS, 0, st>>>(RED_BLOCKS, L.parts, L.scal + 10);
    QES_LAUNCH_CHECK_N(2);
    QES_CUDA_CHECK(cudaMemcpyAsync(&true_rr, L.scal + 10, sizeof(double), cudaMemcpyDeviceToHost, st));
    if ((rc = sr_check_status(L, st))) return rc;        // synchronises the stream
  }
  // x_out = rhs_prefactor * x
  QES_CUDA_CHECK(cudaMemcpyAsync(x_out, x, P * sizeof(V), cudaMemcpyDeviceToDevice, st));
  if (opt->rhs_prefactor != 1.0) {
    scale_vec_kernel<V><<<RED_BLOCKS, RED_THREADS, 0, st>>>(P, opt->rhs_prefactor, x_out);
    QES_LAUNCH_CHECK();
  }
  if (res) {
    res->iterations = (int)hs[5];
    res->converged = done ? 1 : 0;
    res->residual = sqrt(hs[2]);                         // ||r|| (scal[0] holds rho = r^H D^-1 r with PCG)
    res->rhs_norm = sqrt(hs[6]);
    res->e_mean_re = hs[12];
    res->e_mean_im = hs[13];
    res->true_residual = true_rr < 0.0 ? -1.0 : (hs[6] > 0.0 ? sqrt(true_rr / hs[6]) : 0.0);
    res->acond = -1.0;
  }
  return done ? QES_OK : QES_ERR_NOT_CONVERGED;
}

extern "C" int qes_sr_solve_cg_weighted(int dtype, int ns, int nh, int64_t n_samples, const uint32_t* bits,
                                        const void* tanh_theta, const void* eloc, const float* probs,
                                        const qes_sr_options* opt, const void* x0, void* x_out,
                                        qes_sr_result* result, void* workspace, size_t workspace_bytes,
                                        void* stream) {
  QES_ARG_CHECK(ns > 0 && nh > 0 && n_samples > 0 && bits && tanh_theta && eloc && opt && x_out,
                "qes_sr_solve_cg: bad args");
  QES_ARG_CHECK(dtype == QES_DTYPE_F32 || dtype == QES_DTYPE_C64, "qes_sr_solve_cg: bad dtype");
  QES_ARG_CHECK(opt->maxiter >= 0 && opt->shift >= 0.0, "qes_sr_solve_cg: bad options");
  QES_ARG_CHECK(opt->precond == QES_PRECOND_NONE || opt->precond == QES_PRECOND_JACOBI,
                "qes_sr_solve_cg: precond must be QES_PRECOND_NONE or QES_PRECOND_JACOBI");
  SRWork L;
  int rc = check_ws(dtype, ns, nh, n_samples, workspace, workspace_bytes, &L);
  if (rc) return rc;
  L.wts = L.tw.wts = probs;
  cudaStream_t st = (cudaStream_t)stream;
  if (dtype == QES_DTYPE_F32)
    return sr_cg_t<float>(ns, nh, n_samples, bits, (const float*)tanh_theta, (const float2*)eloc, opt,
                          (double*)x_out, result, L, st, (const double*)x0);
  return sr_cg_t<float2>(ns, nh, n_samples, bits, (const float2*)tanh_theta, (const float2*)eloc, opt,
                         (double2*)x_out, result, L, st, (const double2*)x0);
}

// MINRES on (S + shift) x = F with the same force, matvec kernels and stopping rule as the CG
// (||r|| <= max(rtol ||b||, atol), ||r|| = phibar of the recurrences); chunks of check_every
// iterations launched directly, one host check per chunk
template <class T>
static int sr_minres_t(int ns, int nh, int64_t n_samples, const uint32_t* bits, const T* tt, const float2* eloc,
                       const qes_sr_options* opt, typename VecT<T>::type* x_out, qes_sr_result* res, const SRWork& L,
                       cudaStream_t st, const typename VecT<T>::type* x0) {
  using V = typename VecT<T>::type;
  const int64_t P = (int64_t)ns + nh + (int64_t)ns * nh;
  V* x = (V*)L.x; V* r1 = (V*)L.r; V* v = (V*)L.p; V* y = (V*)L.Ap; V* b = (V*)L.b;
  V* r2 = (V*)L.mr2; V* w1 = (V*)L.mw1; V* w2 = (V*)L.mw2;
  int rc = sr_prepare(ScalarTraits<T>::is_complex ? QES_DTYPE_C64 : QES_DTYPE_F32, n_samples, bits, tt, L, st);
  if (rc) return rc;
  rc = sr_force_t<T>(ns, nh, n_samples, bits, tt, eloc, b, L, st);
  if (rc) return rc;
  double emean[2] = {0, 0};
  QES_CUDA_CHECK(cudaMemcpyAsync(emean, L.wmean, 2 * sizeof(double), cudaMemcpyDeviceToHost, st));
  QES_CUDA_CHECK(cudaMemsetAsync(L.counter, 0, 128 * sizeof(unsigned int), st));
  if (x0) {
    QES_CUDA_CHECK(cudaMemcpyAsync(x, x0, P * sizeof(V), cudaMemcpyDeviceToDevice, st));
    rc = sr_matvec_t<T>(ns, nh, n_samples, bits, tt, opt->shift, x, y, nullptr, L, st, false);
    if (rc) return rc;
  }
  minres_init_kernel<V><<<RED_BLOCKS, RED_THREADS, 0, st>>>(P, b, y, x, r1, r2, w1, w2, x0 != nullptr);
  norm2_kernel<V><<<RED_BLOCKS, RED_THREADS, 0, st>>>(P, b, L.parts);
  norm2_kernel<V><<<RED_BLOCKS, RED_THREADS, 0, st>>>(P, r2, L.parts + RED_BLOCKS);
  minres_setup_kernel<<<1, SC_THREADS, 0, st>>>(RED_BLOCKS, L.parts, L.parts + RED_BLOCKS, opt->rtol, opt->atol, L.scal,
                                               L.mscal);
  minres_v_kernel<V><<<RED_BLOCKS, RED_THREADS, 0, st>>>(P, r2, v, L.mscal, L.td, (uint16_t*)nullptr);
  QES_LAUNCH_CHECK_N(5);
  const int check = opt->check_every > 0 ? opt->check_every : 8;
  double hs[8] = {0};
  QES_CUDA_CHECK(cudaMemcpyAsync(hs, L.scal, 8 * sizeof(double), cudaMemcpyDeviceToHost, st));
  QES_CUDA_CHECK(cudaStreamSynchronize(st));
  bool done = hs[4] != 0.0;
  int it = 0;
  while (!done && it < opt->maxiter) {
    const int nrun = std::min(check, opt->maxiter - it);
    for (int q = 0; q < nrun; ++q) {
      // y = (S + shift) v and alpha = v^H y (the split reduction's last block: scal[1])
      rc = sr_matvec_t<T>(ns, nh, n_samples, bits, tt, opt->shift, v, y, L.parts, L, st, /*vp_ready=*/it + q > 0,
                          L.scal + 4);
      if (rc) return rc;
      QES_CUDA_CHECK(qes_launch_pdl(minres_lanczos_kernel<V>, dim3(vec_blocks(P)), dim3(RED_THREADS), 0, st, P,
                                    (const V*)y, r1, r2, L.scal, L.mscal, L.parts, L.counter + 1));
      QES_CUDA_CHECK(qes_launch_pdl(minres_update_kernel<V>, dim3(vec_blocks(P)), dim3(RED_THREADS), 0, st, P, v, w1,
                                    w2, x, (const V*)r2, L.scal, (const double*)L.mscal, L.counter + 2, L.td,
                                    L.tc ? L.tw.vp : (uint16_t*)nullptr));
      QES_LAUNCH_CHECK_N(2);
    }
    it += nrun;
    QES_CUDA_CHECK(cudaMemcpyAsync(hs, L.scal, 8 * sizeof(double), cudaMemcpyDeviceToHost, st));
    if ((rc = sr_check_status(L, st, true))) return rc;     // synchronises the stream
    done = hs[4] != 0.0;
  }
  if ((rc = sr_check_status(L, st, true))) return rc;
  double ms[16] = {0};
  QES_CUDA_CHECK(cudaMemcpyAsync(ms, L.mscal, 16 * sizeof(double), cudaMemcpyDeviceToHost, st));
  double true_rr = -1.0;
  if (opt->maxiter > 0 && !opt->skip_true_residual) {
    rc = sr_matvec_t<T>(ns, nh, n_samples, bits, tt, opt->shift, x, y, nullptr, L, st, false);
    if (rc) return rc;
    diff_norm2_kernel<V><<<RED_BLOCKS, RED_THREADS, 0, st>>>(P, b, y, L.parts);
    sum_parts_kernel<<<1, SC_THREADS, 0, st>>>(RED_BLOCKS, L.parts, L.scal + 10);
    QES_LAUNCH_CHECK_N(2);
    QES_CUDA_CHECK(cudaMemcpyAsync(&true_rr, L.scal + 10, sizeof(double), cudaMemcpyDeviceToHost, st));
  }
  if ((rc = sr_check_status(L, st))) return rc;            // synchronises the stream
  QES_CUDA_CHECK(cudaMemcpyAsync(x_out, x, P * sizeof(V), cudaMemcpyDeviceToDevice, st));
  if (opt->rhs_prefactor != 1.0) {
    scale_vec_kernel<V><<<RED_BLOCKS, RED_THREADS, 0, st>>>(P, opt->rhs_prefactor, x_out);
    QES_LAUNCH_CHECK();
  }
  if (res) {
    res->iterations = (int)hs[5];
    res->converged = done ? 1 : 0;
    res->residual = sqrt(hs[2]);
    res->rhs_norm = sqrt(hs[6]);
    res->e_mean_re = emean[0];
    res->e_mean_im = emean[1];
    res->true_residual = true_rr < 0.0 ? -1.0 : (hs[6] > 0.0 ? sqrt(true_rr / hs[6]) : 0.0);
    res->acond = (ms[13] > 0.0 && ms[13] < 1e300) ? ms[12] / ms[13] : -1.0;
  }
  return done ? QES_OK : QES_ERR_NOT_CONVERGED;
}

extern "C" int qes_sr_solve_minres_weighted(int dtype, int ns, int nh, int64_t n_samples, const uint32_t* bits,
                                            const void* tanh_theta, const void* eloc, const float* probs,
                                            const qes_sr_options* opt, const void* x0, void* x_out,
                                            qes_sr_result* result, void* workspace, size_t workspace_bytes,
                                            void* stream) {
  QES_ARG_CHECK(ns > 0 && nh > 0 && n_samples > 0 && bits && tanh_theta && eloc && opt && x_out,
                "qes_sr_solve_minres: bad args");
  QES_ARG_CHECK(dtype == QES_DTYPE_F32 || dtype == QES_DTYPE_C64, "qes_sr_solve_minres: bad dtype");
  QES_ARG_CHECK(opt->maxiter >= 0 && opt->shift >= 0.0, "qes_sr_solve_minres: bad options");
  QES_ARG_CHECK(opt->precond == QES_PRECOND_NONE, "qes_sr_solve_minres: no preconditioner on the MINRES path");
  SRWork L;
  int rc = check_ws(dtype, ns, nh, n_samples, workspace, workspace_bytes, &L);
  if (rc) return rc;
  L.wts = L.tw.wts = probs;
  cudaStream_t st = (cudaStream_t)stream;
  if (dtype == QES_DTYPE_F32)
    return sr_minres_t<float>(ns, nh, n_samples, bits, (const float*)tanh_theta, (const float2*)eloc, opt,
                              (double*)x_out, result, L, st, (const double*)x0);
  return sr_minres_t<float2>(ns, nh, n_samples, bits, (const float2*)tanh_theta, (const float2*)eloc, opt,
                             (double2*)x_out, result, L, st, (const double2*)x0);
}

extern "C" int qes_sr_solve_cg_x0(int dtype, int ns, int nh, int64_t n_samples, const uint32_t* bits,
                                  const void* tanh_theta, const void* eloc, const qes_sr_options* opt,
                                  const void* x0, void* x_out, qes_sr_result* result, void* workspace,
                                  size_t workspace_bytes, void* stream) {
  return qes_sr_solve_cg_weighted(dtype, ns, nh, n_samples, bits, tanh_theta, eloc, nullptr, opt, x0, x_out, result,
                                  workspace, workspace_bytes, stream);
}

extern "C" int qes_sr_solve_cg(int dtype, int ns, int nh, int64_t n_samples, const uint32_t* bits,
                               const void* tanh_theta, const void* eloc, const qes_sr_options* opt, void* x_out,
                               qes_sr_result* result, void* workspace, size_t workspace_bytes, void* stream) {
  return qes_sr_solve_cg_x0(dtype, ns, nh, n_samples, bits, tanh_theta, eloc, opt, nullptr, x_out, result, workspace,
                            workspace_bytes, stream);
}

// ----------------------------------------------------------------------------
// MinSR (QES/NQS/src/tdvp.py:1199-1226, 1393-1408): solve (T + shift) y = E_c / Ns
// in sample space, T = O_c O_c^H / Ns, and return x = O_c^H y.  Matrix-free with
// the same two contractions in the opposite order: T y = (O g - mean(O g)) / Ns
// with g = O^H (y - mean y).  CG in float64 over Ns-vectors; by the
// push-through identity x equals the parameter-space SR solution.
// ----------------------------------------------------------------------------
// b_s = (E_s - mean E) / n  (real part for a real RBM)
template <class V>
__global__ void minsr_rhs_kernel(int64_t n, const float2* __restrict__ e, const double* __restrict__ mean,
                                 V* __restrict__ b) {
  const double mr = mean[0], mi = mean[1];
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
    if constexpr (sizeof(V) == sizeof(double2)) {
      V v; v.x = ((double)e[k].x - mr) / (double)n; v.y = ((double)e[k].y - mi) / (double)n;
      b[k] = v;
    } else {
      b[k] = ((double)e[k].x - mr) / (double)n;
    }
  }
}

// float32 copy of an Ns-vector (input of the O^H u stage)
template <class V>
__global__ void vec_to_f2_kernel(int64_t n, const V* __restrict__ v, float2* __restrict__ out) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
    if constexpr (sizeof(V) == sizeof(double2)) out[k] = make_float2((float)v[k].x, (float)v[k].y);
    else out[k] = make_float2((float)v[k], 0.f);
  }
}

// Ap = (w - mean w) / n + shift p ; dot partials of p^H Ap, last block: pAp, alpha
template <class V>
__global__ void __launch_bounds__(RED_THREADS) minsr_ap_kernel(int64_t n, const float2* __restrict__ w,
                                                              const double* __restrict__ wmean, double shift,
                                                              const V* __restrict__ p, V* __restrict__ Ap,
                                                              double* __restrict__ dot_part, double* __restrict__ scal,
                                                              unsigned int* __restrict__ counter) {
  const double mr = wmean[0], mi = wmean[1];
  double d = 0.0;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
    V a;
    if constexpr (sizeof(V) == sizeof(double2)) {
      a.x = ((double)w[k].x - mr) / (double)n + shift * p[k].x;
      a.y = ((double)w[k].y - mi) / (double)n + shift * p[k].y;
    } else {
      a = ((double)w[k].x - mr) / (double)n + shift * p[k];
    }
    Ap[k] = a;
    d += vdotc(p[k], a);
  }
  __shared__ double red[RED_THREADS / 32];
  d = warp_sum(d);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = d;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0;
    for (int q = 0; q < RED_THREADS / 32; ++q) t += red[q];
    dot_part[blockIdx.x] = t;
  }
  __shared__ bool last;
  if (threadIdx.x == 0) {            // only thread 0 wrote this block's partial
    __threadfence();
    last = (atomicAdd(counter, 1u) == gridDim.x - 1);
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  double v = 0.0;
  for (int q = threadIdx.x; q < (int)gridDim.x; q += blockDim.x) v += ((volatile double*)dot_part)[q];
  v = warp_sum(v);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double pap = 0.0;
    for (int q = 0; q < RED_THREADS / 32; ++q) pap += red[q];
    scal[1] = pap;
    scal[7] = (scal[4] == 0.0 && pap > 0.0) ? scal[0] / pap : 0.0;
    *counter = 0u;
  }
}

struct MinSRWork {
  float2* uf;      // [Ns] float32 copy of the sample-space vector
  double* umean;   // [2]
  void* g;         // [P] of V
  void *y, *r, *p, *Ap, *b;   // [Ns] of V each
};

static size_t minsr_layout(int dtype, int ns, int nh, int64_t n, char* base, MinSRWork* M) {
  const int64_t P = (int64_t)ns + nh + (int64_t)ns * nh;
  const size_t vs = (dtype == QES_DTYPE_C64) ? sizeof(double2) : sizeof(double);
  const size_t head = sr_layout(dtype, ns, nh, n, nullptr).total;
  size_t off = head;
  auto take = [&](size_t bytes) { char* q = base ? base + off : nullptr; off += align256(bytes); return q; };
  MinSRWork W;
  W.uf = (float2*)take((size_t)n * sizeof(float2));
  W.umean = (double*)take(4 * sizeof(double));
  W.g = take((size_t)P * vs);
  W.y = take((size_t)n * vs);
  W.r = take((size_t)n * vs);
  W.p = take((size_t)n * vs);
  W.Ap = take((size_t)n * vs);
  W.b = take((size_t)n * vs);
  if (M) *M = W;
  return off;
}

extern "C" int qes_sr_minsr_workspace_bytes(int dtype, int ns, int nh, int64_t n_samples, size_t* bytes) {
  QES_ARG_CHECK(bytes && ns > 0 && nh > 0 && n_samples > 0, "qes_sr_minsr_workspace_bytes: bad args");
  *bytes = minsr_layout(dtype, ns, nh, n_samples, nullptr, nullptr);
  return QES_OK;
}

// g = O^H (u - mean u) for a sample-space float64 vector u (tensor cores or CUDA cores)
template <class T>
static int minsr_ohu(int ns, int nh, int64_t n, const uint32_t* bits, const T* tt, const typename VecT<T>::type* u,
                     typename VecT<T>::type* g, const SRWork& L, const MinSRWork& M, cudaStream_t st) {
  using V = typename VecT<T>::type;
  vec_to_f2_kernel<V><<<RED_BLOCKS, RED_THREADS, 0, st>>>(n, u, M.uf);
  mean_c_kernel<<<1, MEAN_THREADS, 0, st>>>(n, M.uf, M.umean);
  QES_LAUNCH_CHECK_N(2);
  if (L.tc) {
    const int dtype = ScalarTraits<T>::is_complex ? QES_DTYPE_C64 : QES_DTYPE_F32;
    int rc = tc_ohu(dtype, L.td, n, M.uf, (const double2*)M.umean, -1, 1.0, L.partial, L.tw, st);
    if (rc) return rc;
    const int64_t P = (int64_t)ns + nh + (int64_t)ns * nh;
    if (int rc_ = launch_reduce_splits<T, V>(P, L.nsplit, L.partial, 0.0,
        nullptr, g, nullptr, nullptr, nullptr, st)) return rc_;
    QES_LAUNCH_CHECK();
    return QES_OK;
  }
  return apply_ohu<T, V>(ns, nh, n, bits, tt, M.uf, M.umean, 1.0, L, 0.0, nullptr, g, nullptr, st);
}

template <class T>
static int sr_minsr_t(int ns, int nh, int64_t n, const uint32_t* bits, const T* tt, const float2* eloc,
                      const qes_sr_options* opt, typename VecT<T>::type* x_out, qes_sr_result* res, const SRWork& L,
                      const MinSRWork& M, cudaStream_t st) {
  using V = typename VecT<T>::type;
  const int dtype = ScalarTraits<T>::is_complex ? QES_DTYPE_C64 : QES_DTYPE_F32;
  const int64_t P = (int64_t)ns + nh + (int64_t)ns * nh;
  V* y = (V*)M.y; V* r = (V*)M.r; V* p = (V*)M.p; V* Ap = (V*)M.Ap; V* b = (V*)M.b; V* g = (V*)M.g;
  QES_ARG_CHECK(!L.fp64, "qes_sr_solve_minsr: the float64 form (impl 3) is not implemented for MinSR");
  int rc = sr_prepare(dtype, n, bits, tt, L, st);
  if (rc) return rc;
  mean_c_kernel<<<1, MEAN_THREADS, 0, st>>>(n, eloc, L.wmean);
  minsr_rhs_kernel<V><<<RED_BLOCKS, RED_THREADS, 0, st>>>(n, eloc, L.wmean, b);
  QES_LAUNCH_CHECK_N(2);
  double emean[2] = {0, 0};
  QES_CUDA_CHECK(cudaMemcpyAsync(emean, L.wmean, 2 * sizeof(double), cudaMemcpyDeviceToHost, st));
  QES_CUDA_CHECK(cudaMemsetAsync(L.counter, 0, 4 * sizeof(unsigned int), st));
  cg_init_kernel<V><<<RED_BLOCKS, RED_THREADS, 0, st>>>(n, b, y, r, p);
  norm2_kernel<V><<<RED_BLOCKS, RED_THREADS, 0, st>>>(n, b, L.parts);
  cg_setup_kernel<<<1, SC_THREADS, 0, st>>>(RED_BLOCKS, L.parts, opt->rtol, opt->atol, L.scal);
  QES_LAUNCH_CHECK_N(3);
  const int check = opt->check_every > 0 ? opt->check_every : 8;
  double hs[8] = {0};
  QES_CUDA_CHECK(cudaMemcpyAsync(hs, L.scal, 8 * sizeof(double), cudaMemcpyDeviceToHost, st));
  QES_CUDA_CHECK(cudaStreamSynchronize(st));
  bool done = hs[4] != 0.0;
  int it = 0;
  while (!done && it < opt->maxiter) {
    const int nrun = std::min(check, opt->maxiter - it);
    for (int q = 0; q < nrun; ++q) {
      if ((rc = minsr_ohu<T>(ns, nh, n, bits, tt, p, g, L, M, st))) return rc;       // g = O_c^H p
      if (L.tc) {                                                                     // w = O g
        if ((rc = tc_ov(dtype, L.td, n, bits, tt, g, L.w, L.tw, st))) return rc;
      } else {
        if ((rc = apply_ov<T, V>(ns, nh, n, bits, tt, g, L.w, nullptr, L, st))) return rc;
      }
      mean_c_kernel<<<1, MEAN_THREADS, 0, st>>>(n, L.w, L.wmean);
      minsr_ap_kernel<V><<<RED_BLOCKS, RED_THREADS, 0, st>>>(n, L.w, L.wmean, opt->shift, p, Ap, L.parts, L.scal,
                                                             L.counter);
      cg_xr_kernel<V><<<vec_blocks(n), RED_THREADS, 0, st>>>(n, p, Ap, y, r, L.scal, L.parts, L.counter + 1);
      cg_p_kernel<V><<<vec_blocks(n), RED_THREADS, 0, st>>>(n, r, p, L.scal, L.td, nullptr);
      QES_LAUNCH_CHECK_N(4);
    }
    it += nrun;
    QES_CUDA_CHECK(cudaMemcpyAsync(hs, L.scal, 8 * sizeof(double), cudaMemcpyDeviceToHost, st));
    if ((rc = sr_check_status(L, st))) return rc;
    done = hs[4] != 0.0;
  }
  // x = rhs_prefactor * O_c^H y
  if ((rc = minsr_ohu<T>(ns, nh, n, bits, tt, y, x_out, L, M, st))) return rc;
  if (opt->rhs_prefactor != 1.0) {
    scale_vec_kernel<V><<<RED_BLOCKS, RED_THREADS, 0, st>>>(P, opt->rhs_prefactor, x_out);
    QES_LAUNCH_CHECK();
  }
  if ((rc = sr_check_status(L, st))) return rc;
  if (res) {
    res->iterations = (int)hs[5];
    res->converged = done ? 1 : 0;
    res->residual = sqrt(hs[4] != 0.0 ? hs[2] : hs[0]);
    res->rhs_norm = sqrt(hs[6]);
    res->e_mean_re = emean[0];
    res->e_mean_im = emean[1];
    res->true_residual = -1.0;                          // not computed for the sample-space solve
    res->acond = -1.0;
  }
  return done ? QES_OK : QES_ERR_NOT_CONVERGED;
}

extern "C" int qes_sr_solve_minsr(int dtype, int ns, int nh, int64_t n_samples, const uint32_t* bits,
                                  const void* tanh_theta, const void* eloc, const qes_sr_options* opt, void* x_out,
                                  qes_sr_result* result, void* workspace, size_t workspace_bytes, void* stream) {
  QES_ARG_CHECK(ns > 0 && nh > 0 && n_samples > 0 && bits && tanh_theta && eloc && opt && x_out,
                "qes_sr_solve_minsr: bad args");
  QES_ARG_CHECK(dtype == QES_DTYPE_F32 || dtype == QES_DTYPE_C64, "qes_sr_solve_minsr: bad dtype");
  QES_ARG_CHECK(opt->maxiter >= 0 && opt->shift >= 0.0, "qes_sr_solve_minsr: bad options");
  QES_ARG_CHECK(opt->precond == QES_PRECOND_NONE, "qes_sr_solve_minsr: no preconditioner on the MinSR system");
  SRWork L;
  int rc = check_ws(dtype, ns, nh, n_samples, workspace, workspace_bytes, &L);
  if (rc) return rc;
  const size_t need = minsr_layout(dtype, ns, nh, n_samples, nullptr, nullptr);
  if (workspace_bytes < need) {
    qes_set_last_message("qes_sr_solve_minsr: workspace too small");
    return QES_ERR_WORKSPACE;
  }
  MinSRWork M;
  minsr_layout(dtype, ns, nh, n_samples, (char*)workspace, &M);
  cudaStream_t st = (cudaStream_t)stream;
  if (dtype == QES_DTYPE_F32)
    return sr_minsr_t<float>(ns, nh, n_samples, bits, (const float*)tanh_theta, (const float2*)eloc, opt,
                             (double*)x_out, result, L, M, st);
  return sr_minsr_t<float2>(ns, nh, n_samples, bits, (const float2*)tanh_theta, (const float2*)eloc, opt,
                            (double2*)x_out, result, L, M, st);
}

// ----------------------------------------------------------------------------
// vector-Jacobian product of log psi:  grad = O^H g  (no centring, no 1/Ns)
// ----------------------------------------------------------------------------
template <class T>
static int vjp_t(int ns, int nh, int64_t n_samples, const uint32_t* bits, const T* tt, const float2* g,
                 typename VecT<T>::type* out, const SRWork& L, cudaStream_t st) {
  using V = typename VecT<T>::type;
  return apply_ohu<T, V>(ns, nh, n_samples, bits, tt, g, nullptr, 1.0, L, 0.0, nullptr, out, nullptr, st);
}

extern "C" int qes_rbm_logpsi_vjp(int dtype, int ns, int nh, int64_t n_samples, const uint32_t* bits,
                                  const void* tanh_theta, const void* g, void* grad_out, void* workspace,
                                  size_t workspace_bytes, void* stream) {
  QES_ARG_CHECK(ns > 0 && nh > 0 && n_samples > 0 && bits && tanh_theta && g && grad_out,
                "qes_rbm_logpsi_vjp: bad args");
  QES_ARG_CHECK(dtype == QES_DTYPE_F32 || dtype == QES_DTYPE_C64, "qes_rbm_logpsi_vjp: bad dtype");
  SRWork L;
  int rc = check_ws(dtype, ns, nh, n_samples, workspace, workspace_bytes, &L);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  if (dtype == QES_DTYPE_F32)
    return vjp_t<float>(ns, nh, n_samples, bits, (const float*)tanh_theta, (const float2*)g, (double*)grad_out, L,
                        st);
  return vjp_t<float2>(ns, nh, n_samples, bits, (const float2*)tanh_theta, (const float2*)g, (double2*)grad_out, L,
                       st);
}

// ----------------------------------------------------------------------------
// Batched problems: one CG per problem, all problems in lockstep launches.
// Per-problem state bscal[b][16]: the CG slots of the single-problem solver
// (0 rr, 1 pAp, 2 rr_new, 3 threshold^2, 4 done, 5 iterations, 6 ||b||^2,
// 7 alpha, 8 beta), 9-10 mean of the current w, 11-12 mean of E_loc.
// Blocks of a converged problem return at once, so its x stays frozen.
// ----------------------------------------------------------------------------
constexpr int BSC = 16;
constexpr int BCG_THREADS = 1024;

QES_D int64_t batch_rows(const qes_batch_instance& I) { return (int64_t)I.n_chains * I.num_samples; }
QES_D int64_t batch_P(const qes_batch_instance& I) { return (int64_t)I.ns + I.nh + (int64_t)I.ns * I.nh; }
QES_D int batch_nsplit(const qes_batch_instance& I) {
  return (int)((batch_rows(I) + OHU_SPLIT_SAMPLES - 1) / OHU_SPLIT_SAMPLES);
}

// fixed-order block sum (valid in every thread)
QES_D double block_allsum(double v, double* red) {
  v = warp_sum(v);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double t = 0.0;
  for (int q = 0; q < (int)(blockDim.x >> 5); ++q) t += red[q];
  return t;
}

// mean of w (or E_loc) rows of problem blockIdx.x -> bscal[b][slot], [slot+1]
__global__ void __launch_bounds__(BCG_THREADS) batch_mean_kernel(const qes_batch_instance* __restrict__ inst,
                                                                const float2* __restrict__ w, double* __restrict__ bscal,
                                                                int slot, int skip_done) {
  const qes_batch_instance I = inst[blockIdx.x];
  double* sc = bscal + (int64_t)blockIdx.x * BSC;
  if (skip_done && sc[4] != 0.0) return;
  const int64_t rows = batch_rows(I);
  const float2* x = w + I.sample_off;
  double sr = 0, si = 0;
  for (int64_t k = threadIdx.x; k < rows; k += blockDim.x) { sr += x[k].x; si += x[k].y; }
  __shared__ double red[BCG_THREADS / 32];
  sr = block_allsum(sr, red);
  si = block_allsum(si, red);
  if (threadIdx.x == 0) {
    sc[slot] = sr / (double)rows;
    sc[slot + 1] = si / (double)rows;
  }
}

// ---- matvec halves of the batched solve (small problems) -------------------------------------
// ov  item (b, first row, rows <= BOV_ROWS, 0): the block stages V = v_W (float32), v_b, v_a and
//     the spins of its rows (as +-1 floats, site-major) in shared memory and computes
//       z_m = v_b,m + sum_i sigma_i V_im ,  (O v)_s = sum_m t_sm z_m + sigma . v_a
//     in 4 x 4 register tiles (batch_ov_tile_kernel below).
// ohu item (b, split z, 0, 0): the block owns every (site, hidden unit) entry of the split's
//     partial, in 4 x 4 register tiles (batch_ohu_tile_kernel below).
constexpr int BOV_ROWS = 64;
// block size limit of the tile kernels (complex tiles hold twice the registers: half the block)
template <class T>
constexpr int bohu_max_threads() { return ScalarTraits<T>::is_complex ? 512 : 1024; }

QES_HD int64_t bsmall_align16(int64_t bytes) { return (bytes + 15) & ~(int64_t)15; }

// ov tiles: thread t owns 4 rows x 4 hidden units (tm = t % n_mt fastest) of
// z_sm = v_b,m + sum_i sigma_si V_im; per site it reads one float4 of signs (4 rows, site-major
// staging) and four V values for 16 multiply-adds, then folds its units into sum_m t_sm z_sm.
// The per-unit-group partial sums meet in shared memory and are added in a fixed order.
QES_HD int bov_round4(int x) { return (x + 3) & ~3; }
template <class T>
QES_HD size_t batch_ov_smem(int ns, int nh) {
  const int nmt = bov_round4(nh) / 4;
  return (size_t)bsmall_align16((int64_t)((int64_t)ns * bov_round4(nh) + bov_round4(nh) + ns) * sizeof(T)) +
         (size_t)bsmall_align16((int64_t)ns * BOV_ROWS * sizeof(float)) + (size_t)BOV_ROWS * nmt * sizeof(T);
}

template <class T, class V>
__global__ void __launch_bounds__(bohu_max_threads<T>()) batch_ov_tile_kernel(const qes_batch_instance* __restrict__ inst,
                                                                             const int4* __restrict__ items,
                                                                             const uint32_t* __restrict__ bits,
                                                                             const T* __restrict__ tt,
                                                                             const V* __restrict__ v,
                                                                             float2* __restrict__ w,
                                                                             const double* __restrict__ bscal) {
  extern __shared__ __align__(16) uint8_t bov_sm[];
  const int4 it = items[blockIdx.x];
  if (bscal[(int64_t)it.x * BSC + 4] != 0.0) return;
  const qes_batch_instance I = inst[it.x];
  const int ns = I.ns, nh = I.nh, nw = n_words(ns);
  const int nhp = bov_round4(nh), nmt = nhp / 4, n_tiles = (BOV_ROWS / 4) * nmt;
  const int64_t r0 = it.y;
  const int nr = it.z;
  T* Vs = reinterpret_cast<T*>(bov_sm);                      // [ns][nhp]
  T* vbs = Vs + (int64_t)ns * nhp;                            // [nhp]
  T* vas = vbs + nhp;                                         // [ns]
  float* sigT = reinterpret_cast<float*>(bov_sm + bsmall_align16((int64_t)((int64_t)ns * nhp + nhp + ns) * sizeof(T)));
  T* red = reinterpret_cast<T*>(reinterpret_cast<uint8_t*>(sigT) + bsmall_align16((int64_t)ns * BOV_ROWS * sizeof(float)));
  const int tid = threadIdx.x, nthr = blockDim.x;
  const V* pv = v + I.param_off;
  {
    const int cm = tid % nhp, ci0 = tid / nhp, cid = nthr / nhp;   // V entry (i, m), divided once
    if (ci0 < cid)
      for (int i = ci0; i < ns; i += cid) Vs[i * nhp + cm] = (cm < nh) ? to_f(pv[ns + nh + (int64_t)i * nh + cm]) : ScalarTraits<T>::zero();
  }
  for (int m = tid; m < nhp; m += nthr) vbs[m] = (m < nh) ? to_f(pv[ns + m]) : ScalarTraits<T>::zero();
  for (int i = tid; i < ns; i += nthr) vas[i] = to_f(pv[i]);
  const uint32_t* bw = bits + I.sample_word_off;
  {
    const int q = tid % BOV_ROWS, i0 = tid / BOV_ROWS, di = nthr / BOV_ROWS;
    for (int i = i0; i < ns; i += di) {
      float sg = 0.f;
      if (q < nr) sg = ((bw[(r0 + q) * nw + (i >> 5)] >> (i & 31)) & 1u) ? 1.f : -1.f;
      sigT[i * BOV_ROWS + q] = sg;
    }
  }
  __syncthreads();
  const T* tb = tt + I.tanh_off;
  for (int t0 = 0; t0 < n_tiles; t0 += nthr) {
    const int t = t0 + tid;
    if (t < n_tiles) {
      const int tm = t % nmt, sg = t / nmt;
      T z[4][4];
#pragma unroll
      for (int b = 0; b < 4; ++b) {
        const T vb = vbs[4 * tm + b];
#pragma unroll
        for (int a = 0; a < 4; ++a) z[a][b] = vb;
      }
      for (int i = 0; i < ns; ++i) {
        const float4 s4 = *reinterpret_cast<const float4*>(sigT + i * BOV_ROWS + 4 * sg);
        const T* vr = Vs + (int64_t)i * nhp + 4 * tm;
        T vv[4];
        if constexpr (ScalarTraits<T>::is_complex) {
          const float4 a01 = reinterpret_cast<const float4*>(vr)[0], a23 = reinterpret_cast<const float4*>(vr)[1];
          vv[0] = make_float2(a01.x, a01.y); vv[1] = make_float2(a01.z, a01.w);
          vv[2] = make_float2(a23.x, a23.y); vv[3] = make_float2(a23.z, a23.w);
        } else {
          const float4 a4 = *reinterpret_cast<const float4*>(vr);
          vv[0] = a4.x; vv[1] = a4.y; vv[2] = a4.z; vv[3] = a4.w;
        }
        const float sv[4] = {s4.x, s4.y, s4.z, s4.w};
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
          for (int b = 0; b < 4; ++b) z[a][b] = addx(z[a][b], scal(sv[a], vv[b]));
      }
#pragma unroll
      for (int a = 0; a < 4; ++a) {
        const int q = 4 * sg + a;
        T acc = ScalarTraits<T>::zero();
        if (q < nr) {
          const T* trow = tb + (r0 + q) * nh;
#pragma unroll
          for (int b = 0; b < 4; ++b) {
            const int m = 4 * tm + b;
            if (m < nh) acc = addx(acc, mulx(trow[m], z[a][b]));
          }
        }
        red[q * nmt + tm] = acc;
      }
    }
  }
  __syncthreads();
  float2* wo = w + I.sample_off;
  for (int q = tid; q < nr; q += nthr) {
    T acc = ScalarTraits<T>::zero();
    for (int g = 0; g < nmt; ++g) acc = addx(acc, red[q * nmt + g]);
    for (int i = 0; i < ns; ++i) acc = addx(acc, scal(sigT[i * BOV_ROWS + q], vas[i]));
    wo[r0 + q] = to_c(acc);
  }
}

// ohu tiles: the split's partial is the (ns + 1) x (nh + 1) matrix  sum_s sigma'_si q'_sm  with a
// virtual site ns (sigma' = 1: row ns is g_b = sum_s q_s) and a virtual hidden unit nh
// (q' = u: column nh is g_a = sum_s sigma_s u_s); entry (ns, nh) is unused.  Thread t owns a
// 4 x 4 tile (sites 4 ti.., units 4 tm..), tm = t % n_mt fastest; per staged sample it reads one
// float4 of signs and four q values from shared memory for 16 multiply-adds.  Tiles beyond the
// block size take further passes over the samples.  (8 x 4 tiles, fewer threads per block, ran
// slower: the staging latency, not the multiply-adds, sets the pace.)

constexpr size_t BOHU_SMEM_TARGET = 200 * 1024;   // up to a whole split (256 samples) staged at once

QES_HD int bohu_round4(int x) { return (x + 3) & ~3; }
QES_HD int batch_ohu_tiles(int ns, int nh) { return (bohu_round4(ns + 1) / 4) * (bohu_round4(nh + 1) / 4); }
// staged samples per pass for rows of (nh + 1) q values and (ns + 1) signs
template <class T>
QES_HD int batch_ohu_sc(int ns_max_row, int nh_max_row) {
  const size_t row = (size_t)bohu_round4(nh_max_row + 1) * sizeof(T) + (size_t)bohu_round4(ns_max_row + 1) * 4;
  int sc = (int)(BOHU_SMEM_TARGET / row);
  sc = sc > OHU_SPLIT_SAMPLES ? OHU_SPLIT_SAMPLES : sc;
  return sc < 4 ? 4 : sc;
}

template <class T>
__global__ void __launch_bounds__(bohu_max_threads<T>()) batch_ohu_tile_kernel(const qes_batch_instance* __restrict__ inst,
                                                                         const int4* __restrict__ items,
                                                                         const uint32_t* __restrict__ bits,
                                                                         const T* __restrict__ tt,
                                                                         const float2* __restrict__ w,
                                                                         const double* __restrict__ bscal, int mslot,
                                                                         int skip_done, int SC, int qstride,
                                                                         int sstride, T* __restrict__ partial) {
  extern __shared__ __align__(16) uint8_t boh_sm[];
  const int4 it = items[blockIdx.x];
  const double* sc = bscal + (int64_t)it.x * BSC;
  if (skip_done && sc[4] != 0.0) return;
  const qes_batch_instance I = inst[it.x];
  const int ns = I.ns, nh = I.nh, nw = n_words(ns);
  const int nsp = bohu_round4(ns + 1), nqp = bohu_round4(nh + 1);
  const int nst = nsp / 4, nmt = nqp / 4, n_tiles = nst * nmt;
  const int64_t rows = batch_rows(I);
  T* Q = reinterpret_cast<T*>(boh_sm);                                       // [SC][qstride]
  float* sig = reinterpret_cast<float*>(boh_sm + bsmall_align16((int64_t)SC * qstride * sizeof(T)));   // [SC][sstride]
  const int tid = threadIdx.x, nthr = blockDim.x;
  const float mr = (float)sc[mslot], mi = (float)sc[mslot + 1];
  const float fs = (float)(1.0 / (double)rows);
  const uint32_t* bw = bits + I.sample_word_off;
  const T* tb = tt + I.tanh_off;
  const float2* wb = w + I.sample_off;
  const int64_t sbeg = (int64_t)it.y * OHU_SPLIT_SAMPLES;
  const int64_t send = min(rows, sbeg + OHU_SPLIT_SAMPLES);
  // staging coordinates, divided once: Q entry (sl, m) and sign entry (sl, i)
  const int qm = tid % nqp, qs0 = tid / nqp, qsd = nthr / nqp;
  const int si = tid % nsp, ss0 = tid / nsp, ssd = nthr / nsp;
  const int64_t P = (int64_t)ns + nh + (int64_t)ns * nh;
  T* out = partial + I.sr_part_off + (int64_t)it.y * P;
  // small problems: the block's threads form G sample groups over the tiles (group g takes the
  // samples g, g + G, ...), summed in a fixed order at the end; large ones take passes over the tiles
  const int G = (n_tiles <= nthr) ? nthr / n_tiles : 1;
  for (int t0 = 0; t0 < n_tiles; t0 += nthr) {
    const int t = (G > 1) ? tid % n_tiles : t0 + tid;
    const int grp = (G > 1) ? tid / n_tiles : 0;
    const bool active = (G > 1) ? grp < G : t < n_tiles;
    const int tm = active ? t % nmt : 0, ti = active ? t / nmt : 0;
    T acc[4][4];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < 4; ++b) acc[a][b] = ScalarTraits<T>::zero();
    for (int64_t c0 = sbeg; c0 < send; c0 += SC) {
      const int nc = (int)min((int64_t)SC, send - c0);
      // staging in batches of SB rows per thread: the global loads of a batch are issued together
      constexpr int SB = ScalarTraits<T>::is_complex ? 8 : 4;   // real: within the 64-register budget
      if (qs0 < qsd) {
        for (int sl0 = qs0; sl0 < SC; sl0 += SB * qsd) {
          T tv[SB];
          float2 wv[SB];
#pragma unroll
          for (int b = 0; b < SB; ++b) {
            const int sl = sl0 + b * qsd;
            const bool ok = sl < nc;
            wv[b] = ok ? wb[c0 + sl] : make_float2(0.f, 0.f);
            tv[b] = (ok && qm < nh) ? tb[(c0 + sl) * nh + qm] : ScalarTraits<T>::zero();
          }
#pragma unroll
          for (int b = 0; b < SB; ++b) {
            const int sl = sl0 + b * qsd;
            if (sl < SC) {
              T q = ScalarTraits<T>::zero();
              if (sl < nc) {
                const T u = from_c(make_float2((wv[b].x - mr) * fs, (wv[b].y - mi) * fs), T());
                if (qm < nh) q = mulx(conjx(tv[b]), u);
                else if (qm == nh) q = u;                                  // virtual unit: g_a
              }
              Q[sl * qstride + qm] = q;
            }
          }
        }
      }
      if (ss0 < ssd) {
        for (int sl0 = ss0; sl0 < SC; sl0 += SB * ssd) {
          uint32_t wd[SB];
#pragma unroll
          for (int b = 0; b < SB; ++b) {
            const int sl = sl0 + b * ssd;
            wd[b] = (sl < nc && si < ns) ? bw[(c0 + sl) * nw + (si >> 5)] : 0u;
          }
#pragma unroll
          for (int b = 0; b < SB; ++b) {
            const int sl = sl0 + b * ssd;
            if (sl < SC) {
              float sg = 0.f;
              if (sl < nc) {
                if (si < ns) sg = ((wd[b] >> (si & 31)) & 1u) ? 1.f : -1.f;
                else if (si == ns) sg = 1.f;                               // virtual site: g_b
              }
              sig[sl * sstride + si] = sg;
            }
          }
        }
      }
      __syncthreads();
      if (active) {
        for (int sl = grp; sl < nc; sl += G) {
          const float4 s4 = *reinterpret_cast<const float4*>(sig + sl * sstride + 4 * ti);
          T q[4];
          if constexpr (ScalarTraits<T>::is_complex) {
            const float4* qr = reinterpret_cast<const float4*>(Q + sl * qstride + 4 * tm);
            const float4 q01 = qr[0], q23 = qr[1];
            q[0] = make_float2(q01.x, q01.y); q[1] = make_float2(q01.z, q01.w);
            q[2] = make_float2(q23.x, q23.y); q[3] = make_float2(q23.z, q23.w);
          } else {
            const float4 q4 = *reinterpret_cast<const float4*>(Q + sl * qstride + 4 * tm);
            q[0] = q4.x; q[1] = q4.y; q[2] = q4.z; q[3] = q4.w;
          }
          const float sv[4] = {s4.x, s4.y, s4.z, s4.w};
#pragma unroll
          for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 4; ++b) acc[a][b] = addx(acc[a][b], scal(sv[a], q[b]));
        }
      }
      __syncthreads();
    }
    if (G > 1) {
      // group partials through shared memory (the staging buffers are free), group 0 adds them
      T* gred = reinterpret_cast<T*>(boh_sm);             // [G][n_tiles][16]
      if (active) {
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
          for (int b = 0; b < 4; ++b) gred[((size_t)grp * n_tiles + t) * 16 + a * 4 + b] = acc[a][b];
      }
      __syncthreads();
      if (active && grp == 0) {
        for (int g = 1; g < G; ++g)
#pragma unroll
          for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 4; ++b) acc[a][b] = addx(acc[a][b], gred[((size_t)g * n_tiles + t) * 16 + a * 4 + b]);
      }
    }
    if (active && grp == 0) {
#pragma unroll
      for (int a = 0; a < 4; ++a) {
        const int i = 4 * ti + a;
#pragma unroll
        for (int b = 0; b < 4; ++b) {
          const int m = 4 * tm + b;
          if (i < ns && m < nh) out[ns + nh + (int64_t)i * nh + m] = acc[a][b];
          else if (i == ns && m < nh) out[ns + m] = acc[a][b];
          else if (i < ns && m == nh) out[i] = acc[a][b];
        }
      }
    }
  }
}

// b = sum of the force partials; x = 0, r = p = b; CG scalars (one block per problem)
template <class T, class V>
__global__ void __launch_bounds__(BCG_THREADS) batch_cg_setup_kernel(const qes_batch_instance* __restrict__ inst,
                                                                    const T* __restrict__ partial, double rtol,
                                                                    double atol, V* __restrict__ x, V* __restrict__ r,
                                                                    V* __restrict__ p, V* __restrict__ bvec,
                                                                    double* __restrict__ bscal,
                                                                    unsigned int* __restrict__ n_done) {
  const qes_batch_instance I = inst[blockIdx.x];
  double* sc = bscal + (int64_t)blockIdx.x * BSC;
  const int64_t P = batch_P(I), o = I.param_off;
  const int nz = batch_nsplit(I);
  const T* part = partial + I.sr_part_off;
  double d = 0.0;
  for (int64_t k = threadIdx.x; k < P; k += blockDim.x) {
    V g = vzero(V());
    for (int z = 0; z < nz; ++z) g = vadd(g, to_d(part[(int64_t)z * P + k]));
    bvec[o + k] = g;
    x[o + k] = vzero(V());
    r[o + k] = g;
    p[o + k] = g;
    d += vdotc(g, g);
  }
  __shared__ double red[BCG_THREADS / 32];
  d = block_allsum(d, red);
  if (threadIdx.x == 0) {
    const double th = fmax(rtol * sqrt(d), atol);
    sc[0] = d; sc[1] = 0.0; sc[2] = d; sc[3] = th * th;
    sc[5] = 0.0; sc[6] = d; sc[7] = 0.0; sc[8] = 0.0;
    sc[11] = sc[9]; sc[12] = sc[10];
    sc[4] = (d <= sc[3]) ? 1.0 : 0.0;
    if (sc[4] != 0.0) atomicAdd(n_done, 1u);
  }
}

// y = sum of the matvec partials + shift p; alpha; x += alpha p; r -= alpha y; beta; p = r + beta p
template <class T, class V>
__global__ void __launch_bounds__(BCG_THREADS) batch_cg_update_kernel(const qes_batch_instance* __restrict__ inst,
                                                                     const T* __restrict__ partial, double shift,
                                                                     V* __restrict__ x, V* __restrict__ r,
                                                                     V* __restrict__ p, V* __restrict__ Ap,
                                                                     double* __restrict__ bscal,
                                                                     unsigned int* __restrict__ n_done) {
  double* sc = bscal + (int64_t)blockIdx.x * BSC;
  if (sc[4] != 0.0) return;
  const qes_batch_instance I = inst[blockIdx.x];
  const int64_t P = batch_P(I), o = I.param_off;
  const int nz = batch_nsplit(I);
  const T* part = partial + I.sr_part_off;
  __shared__ double red[BCG_THREADS / 32];
  double d = 0.0;
  // the split loads of an element are issued together (fixed summation order)
  for (int64_t k = threadIdx.x; k < P; k += blockDim.x) {
    const V pk = p[o + k];
    V g = vzero(V());
    int z = 0;
    for (; z + 8 <= nz; z += 8) {
      T q[8];
#pragma unroll
      for (int b = 0; b < 8; ++b) q[b] = part[(int64_t)(z + b) * P + k];
#pragma unroll
      for (int b = 0; b < 8; ++b) g = vadd(g, to_d(q[b]));
    }
    for (; z < nz; ++z) g = vadd(g, to_d(part[(int64_t)z * P + k]));
    g = vadd(g, vscale(shift, pk));
    Ap[o + k] = g;
    d += vdotc(pk, g);
  }
  const double pap = block_allsum(d, red);
  const double alpha = (pap > 0.0) ? sc[0] / pap : 0.0;
  double e = 0.0;
  for (int64_t k = threadIdx.x; k < P; k += blockDim.x) {
    x[o + k] = vadd(x[o + k], vscale(alpha, p[o + k]));
    const V rk = vadd(r[o + k], vscale(-alpha, Ap[o + k]));
    r[o + k] = rk;
    e += vdotc(rk, rk);
  }
  const double rr_new = block_allsum(e, red);
  const double beta = (sc[0] > 0.0) ? rr_new / sc[0] : 0.0;
  const bool conv = rr_new <= sc[3];
  if (!conv)
    for (int64_t k = threadIdx.x; k < P; k += blockDim.x) p[o + k] = vadd(r[o + k], vscale(beta, p[o + k]));
  __syncthreads();
  if (threadIdx.x == 0) {
    sc[1] = pap; sc[7] = alpha; sc[2] = rr_new; sc[8] = beta; sc[0] = rr_new;
    sc[5] += 1.0;
    if (conv) {
      sc[4] = 1.0;
      atomicAdd(n_done, 1u);
    }
  }
}

struct BatchSRWork {
  double* bscal;        // [n_inst][BSC]
  unsigned int* n_done; // [1] (+pad)
  float2* w;            // [n_samples_total]
  void* partial;        // [sr_part_total] of T
  void *r, *p, *Ap, *b; // [n_params_total] of V each
};

static size_t batch_sr_layout(int dtype, int n_inst, int64_t n_params_total, int64_t n_samples_total,
                              int64_t sr_part_total, char* base, BatchSRWork* L) {
  const size_t ts = (dtype == QES_DTYPE_C64) ? sizeof(float2) : sizeof(float);
  const size_t vs = (dtype == QES_DTYPE_C64) ? sizeof(double2) : sizeof(double);
  auto up = [](size_t v) { return (v + 255) & ~(size_t)255; };
  size_t off = 0;
  auto take = [&](size_t bytes) { char* q = base ? base + off : nullptr; off += up(bytes); return q; };
  BatchSRWork W;
  W.bscal = (double*)take((size_t)n_inst * BSC * sizeof(double));
  W.n_done = (unsigned int*)take(256);
  W.w = (float2*)take((size_t)n_samples_total * sizeof(float2));
  W.partial = take((size_t)sr_part_total * ts);
  W.r = take((size_t)n_params_total * vs);
  W.p = take((size_t)n_params_total * vs);
  W.Ap = take((size_t)n_params_total * vs);
  W.b = take((size_t)n_params_total * vs);
  if (L) *L = W;
  return off;
}

extern "C" int qes_batch_sr_workspace_bytes(int dtype, int n_inst, int64_t n_params_total, int64_t n_samples_total,
                                            int64_t sr_part_total, size_t* bytes) {
  QES_ARG_CHECK(bytes && n_inst >= 0 && n_params_total >= 0 && n_samples_total >= 0 && sr_part_total >= 0,
                "qes_batch_sr_workspace_bytes: bad args");
  *bytes = batch_sr_layout(dtype, n_inst, n_params_total, n_samples_total, sr_part_total, nullptr, nullptr);
  return QES_OK;
}

template <class T, class V>
static int launch_batch_ov(int n_ov, int threads, size_t smem, const qes_batch_instance* inst, const int4* items,
                           const uint32_t* bits, const T* tt, const V* p, float2* w, const double* bscal,
                           cudaStream_t st) {
  QES_CUDA_CHECK(cudaFuncSetAttribute(batch_ov_tile_kernel<T, V>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)smem));
  const int pf = qes_prof_begin(QES_PROF_OV, st);
  batch_ov_tile_kernel<T, V><<<n_ov, threads, smem, st>>>(inst, items, bits, tt, p, w, bscal);
  qes_prof_end(pf, st);
  return QES_OK;
}

template <class T>
static int launch_batch_ohu(int n_ohu, int threads, int SC, int qstride, int sstride, size_t smem,
                            const qes_batch_instance* inst, const int4* items, const uint32_t* bits, const T* tt,
                            const float2* w, const double* bscal, int skip_done, T* partial, cudaStream_t st) {
  QES_CUDA_CHECK(cudaFuncSetAttribute(batch_ohu_tile_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)smem));
  const int pf = qes_prof_begin(QES_PROF_OHU, st);
  batch_ohu_tile_kernel<T><<<n_ohu, threads, smem, st>>>(inst, items, bits, tt, w, bscal, 9, skip_done, SC, qstride,
                                                         sstride, partial);
  qes_prof_end(pf, st);
  return QES_OK;
}

struct BatchGraphKey {
  const void* inst; const void* ov_items; const void* ohu_items; const void* bits; const void* tt; const void* x;
  const void* bscal;
  int n_inst, n_ov, n_ohu, chunk, cplx, ov_threads, ohu_threads, ohu_sc, ohu_qstride, ohu_sstride, pad0, pad1;
  int64_t ov_smem, ohu_smem;
  double shift;
  bool operator==(const BatchGraphKey& o) const { return std::memcmp(this, &o, sizeof(*this)) == 0; }
};
static_assert(sizeof(BatchGraphKey) == 7 * sizeof(void*) + 12 * 4 + 2 * 8 + 8, "BatchGraphKey has padding bytes");
struct BatchGraphSlot {
  bool init = false;
  cudaStream_t cs = nullptr;
  cudaEvent_t ev_in = nullptr, ev_out = nullptr;
  cudaGraphExec_t exec = nullptr;
  BatchGraphKey key{};
  long long nodes = 0;
};
static std::mutex g_bgraph_mu;
static BatchGraphSlot g_bgraph[kMaxGraphDevices];

template <class T>
static int batch_sr_cg_t(int n_inst, const qes_batch_instance* inst, int n_ov, const int4* ov_items, int n_ohu,
                         const int4* ohu_items, int64_t n_params_total, const uint32_t* bits, const T* tt,
                         const float2* eloc, const qes_sr_options* opt, typename VecT<T>::type* x,
                         qes_sr_result* res, const BatchSRWork& L, cudaStream_t st) {
  using V = typename VecT<T>::type;
  constexpr bool CPLX = ScalarTraits<T>::is_complex;
  T* partial = (T*)L.partial;
  V* r = (V*)L.r; V* p = (V*)L.p; V* Ap = (V*)L.Ap; V* b = (V*)L.b;
  // the shapes pick the kernel variants: read the descriptors once
  std::vector<qes_batch_instance> hi(n_inst);
  QES_CUDA_CHECK(cudaMemcpyAsync(hi.data(), inst, n_inst * sizeof(qes_batch_instance), cudaMemcpyDeviceToHost, st));
  QES_CUDA_CHECK(cudaStreamSynchronize(st));
  int max_nh = 1, max_ns = 1, max_tiles = 1;
  size_t ov_smem = 0;
  for (const auto& d : hi) {
    if (d.ns <= 0 || d.nh <= 0 || d.nh > 512 || d.ns >= 512 || (int64_t)d.ns * d.nh > (CPLX ? 8192 : 16384)) {
      qes_set_last_message("qes_batch_sr_solve_cg: a problem exceeds ns*nh <= 16384 (real) / 8192 (complex), "
                           "nh <= 512");
      return QES_ERR_SIZE;
    }
    max_nh = std::max(max_nh, d.nh);
    max_ns = std::max(max_ns, d.ns);
    max_tiles = std::max(max_tiles, batch_ohu_tiles(d.ns, d.nh));
    ov_smem = std::max(ov_smem, batch_ov_smem<T>(d.ns, d.nh));
  }
  // O^H u: one block size for every split (enough threads for the largest problem's tiles)
  const int ohu_qstride = bohu_round4(max_nh + 1), ohu_sstride = bohu_round4(max_ns + 1);
  // at least one thread per staged row entry (q values and signs), at most 1024 (real) / 512
  // (complex); tiles beyond take further passes
  const int ohu_threads =
      std::min(bohu_max_threads<T>(), (std::max({max_tiles, ohu_qstride, ohu_sstride}) + 31) / 32 * 32);
  const int ohu_sc = batch_ohu_sc<T>(max_ns, max_nh);
  const size_t ohu_smem = std::max((size_t)bsmall_align16((int64_t)ohu_sc * ohu_qstride * sizeof(T)) +
                                       (size_t)ohu_sc * ohu_sstride * sizeof(float),
                                   (size_t)ohu_threads * 16 * sizeof(T));      // sample-group partials
  // O v: enough threads for the staging rows (BOV_ROWS signs, nh + ... V columns) and the tiles
  const int ov_threads = std::min(bohu_max_threads<T>(),
                                  (std::max({(BOV_ROWS / 4) * (bov_round4(max_nh) / 4), bov_round4(max_nh), BOV_ROWS}) +
                                   31) / 32 * 32);
  auto ov = [&](const V* vec) -> int {
    return launch_batch_ov<T, V>(n_ov, ov_threads, ov_smem, inst, ov_items, bits, tt, vec, L.w, L.bscal, st);
  };
  auto ohu = [&](const float2* g, int skip) -> int {
    return launch_batch_ohu<T>(n_ohu, ohu_threads, ohu_sc, ohu_qstride, ohu_sstride, ohu_smem, inst, ohu_items, bits,
                               tt, g, L.bscal, skip, partial, st);
  };
  int rc;
  QES_CUDA_CHECK(cudaMemsetAsync(L.n_done, 0, sizeof(unsigned int), st));
  // force: mean of E_loc, O^H (E - mean) / rows, then CG set-up
  batch_mean_kernel<<<n_inst, BCG_THREADS, 0, st>>>(inst, eloc, L.bscal, 9, 0);
  if ((rc = ohu(eloc, 0))) return rc;
  batch_cg_setup_kernel<T, V><<<n_inst, BCG_THREADS, 0, st>>>(inst, partial, opt->rtol, opt->atol, x, r, p, b,
                                                              L.bscal, L.n_done);
  QES_LAUNCH_CHECK_N(3);
  const int check = opt->check_every > 0 ? opt->check_every : 8;
  unsigned int done = 0;
  QES_CUDA_CHECK(cudaMemcpyAsync(&done, L.n_done, sizeof(unsigned int), cudaMemcpyDeviceToHost, st));
  QES_CUDA_CHECK(cudaStreamSynchronize(st));
  int it = 0;
  auto run_chunk = [&](int nrun) -> int {
    for (int q = 0; q < nrun; ++q) {
      int r2;
      if ((r2 = ov(p))) return r2;
      batch_mean_kernel<<<n_inst, BCG_THREADS, 0, st>>>(inst, L.w, L.bscal, 9, 1);
      if ((r2 = ohu(L.w, 1))) return r2;
      const int pfr = qes_prof_begin(QES_PROF_REDUCE, st);
      batch_cg_update_kernel<T, V><<<n_inst, BCG_THREADS, 0, st>>>(inst, partial, opt->shift, x, r, p, Ap, L.bscal,
                                                                   L.n_done);
      qes_prof_end(pfr, st);
      QES_LAUNCH_CHECK_N(4);
    }
    return QES_OK;
  };
  // Full chunks run as one CUDA graph on a private stream (captured once per launch configuration
  // and set of buffers, then replayed): four launches per lockstep iteration otherwise
  int dev = 0;
  QES_CUDA_CHECK(cudaGetDevice(&dev));
  const bool graphs = g_use_graphs.load() != 0 && !qes_prof_on() && dev >= 0 && dev < kMaxGraphDevices;
  while ((int)done < n_inst && it < opt->maxiter) {
    const int nrun = std::min(check, opt->maxiter - it);
    if (!graphs || nrun != check) {
      if ((rc = run_chunk(nrun))) return rc;
    } else {
      std::lock_guard<std::mutex> lock(g_bgraph_mu);
      BatchGraphSlot& gs = g_bgraph[dev];
      if (!gs.init) {
        QES_CUDA_CHECK(cudaStreamCreateWithFlags(&gs.cs, cudaStreamNonBlocking));
        QES_CUDA_CHECK(cudaEventCreateWithFlags(&gs.ev_in, cudaEventDisableTiming));
        QES_CUDA_CHECK(cudaEventCreateWithFlags(&gs.ev_out, cudaEventDisableTiming));
        gs.init = true;
      }
      const BatchGraphKey key{inst, ov_items, ohu_items, bits, tt, x, L.bscal, n_inst, n_ov, n_ohu, nrun,
                              CPLX ? 1 : 0, ov_threads, ohu_threads, ohu_sc, ohu_qstride, ohu_sstride, 0, 0,
                              (int64_t)ov_smem, (int64_t)ohu_smem, opt->shift};
      if (gs.exec == nullptr || !(gs.key == key)) {
        if (gs.exec) {
          cudaGraphExecDestroy(gs.exec);
          gs.exec = nullptr;
        }
        const long long before = qes_launch_count(0);
        QES_CUDA_CHECK(cudaStreamBeginCapture(gs.cs, cudaStreamCaptureModeThreadLocal));
        cudaStream_t saved = st;
        st = gs.cs;
        const int rcap = run_chunk(nrun);
        st = saved;
        cudaGraph_t g = nullptr;
        const cudaError_t ec = cudaStreamEndCapture(gs.cs, &g);
        if (rcap) return rcap;
        if (ec != cudaSuccess) { qes_set_last_error(ec, "cudaStreamEndCapture"); return QES_ERR_CUDA; }
        const cudaError_t ei = cudaGraphInstantiate(&gs.exec, g, 0);
        cudaGraphDestroy(g);
        if (ei != cudaSuccess) { gs.exec = nullptr; qes_set_last_error(ei, "cudaGraphInstantiate"); return QES_ERR_CUDA; }
        gs.nodes = qes_launch_count(0) - before;
        qes_count_launches((int)-gs.nodes);     // captured, not run
        gs.key = key;
      }
      QES_CUDA_CHECK(cudaEventRecord(gs.ev_in, st));
      QES_CUDA_CHECK(cudaStreamWaitEvent(gs.cs, gs.ev_in, 0));
      QES_CUDA_CHECK(cudaGraphLaunch(gs.exec, gs.cs));
      QES_CUDA_CHECK(cudaEventRecord(gs.ev_out, gs.cs));
      QES_CUDA_CHECK(cudaStreamWaitEvent(st, gs.ev_out, 0));
      qes_count_launches((int)gs.nodes);
    }
    it += nrun;
    QES_CUDA_CHECK(cudaMemcpyAsync(&done, L.n_done, sizeof(unsigned int), cudaMemcpyDeviceToHost, st));
    QES_CUDA_CHECK(cudaStreamSynchronize(st));
  }
  if (opt->rhs_prefactor != 1.0) {
    scale_vec_kernel<V><<<RED_BLOCKS, RED_THREADS, 0, st>>>(n_params_total, opt->rhs_prefactor, x);
    QES_LAUNCH_CHECK();
  }
  if (res) {
    std::vector<double> hs((size_t)n_inst * BSC);
    QES_CUDA_CHECK(cudaMemcpyAsync(hs.data(), L.bscal, hs.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    QES_CUDA_CHECK(cudaStreamSynchronize(st));
    for (int q = 0; q < n_inst; ++q) {
      const double* h = hs.data() + (size_t)q * BSC;
      res[q].iterations = (int)h[5];
      res[q].converged = h[4] != 0.0 ? 1 : 0;
      res[q].residual = sqrt(h[0]);
      res[q].rhs_norm = sqrt(h[6]);
      res[q].e_mean_re = h[11];
      res[q].e_mean_im = h[12];
    }
  }
  return (int)done == n_inst ? QES_OK : QES_ERR_NOT_CONVERGED;
}

extern "C" int qes_batch_sr_solve_cg(int dtype, int n_inst, const qes_batch_instance* inst, int n_ov_items,
                                     const int32_t* ov_items, int n_ohu_items, const int32_t* ohu_items,
                                     int64_t n_params_total, int64_t n_samples_total, int64_t sr_part_total,
                                     const uint32_t* sample_bits, const void* tanh_theta, const void* eloc,
                                     const qes_sr_options* opts, void* x_out, qes_sr_result* results,
                                     void* workspace, size_t workspace_bytes, void* stream) {
  QES_ARG_CHECK(dtype == QES_DTYPE_F32 || dtype == QES_DTYPE_C64, "qes_batch_sr_solve_cg: bad dtype");
  QES_ARG_CHECK(n_inst > 0 && n_ov_items > 0 && n_ohu_items > 0 && n_params_total > 0 && n_samples_total > 0,
                "qes_batch_sr_solve_cg: bad sizes");
  QES_ARG_CHECK(inst && ov_items && ohu_items && sample_bits && tanh_theta && eloc && opts && x_out,
                "qes_batch_sr_solve_cg: null pointer");
  QES_ARG_CHECK(opts->maxiter >= 0 && opts->shift >= 0.0, "qes_batch_sr_solve_cg: bad options");
  QES_ARG_CHECK(opts->precond == QES_PRECOND_NONE, "qes_batch_sr_solve_cg: no preconditioner on the batched CG");
  const size_t need = batch_sr_layout(dtype, n_inst, n_params_total, n_samples_total, sr_part_total, nullptr, nullptr);
  if (!workspace || workspace_bytes < need) {
    qes_set_last_message("qes_batch_sr_solve_cg: workspace too small");
    return QES_ERR_WORKSPACE;
  }
  BatchSRWork L;
  batch_sr_layout(dtype, n_inst, n_params_total, n_samples_total, sr_part_total, (char*)workspace, &L);
  cudaStream_t st = (cudaStream_t)stream;
  if (dtype == QES_DTYPE_F32)
    return batch_sr_cg_t<float>(n_inst, inst, n_ov_items, (const int4*)ov_items, n_ohu_items, (const int4*)ohu_items,
                                n_params_total, sample_bits, (const float*)tanh_theta, (const float2*)eloc, opts,
                                (double*)x_out, results, L, st);
  return batch_sr_cg_t<float2>(n_inst, inst, n_ov_items, (const int4*)ov_items, n_ohu_items, (const int4*)ohu_items,
                               n_params_total, sample_bits, (const float2*)tanh_theta, (const float2*)eloc, opts,
                               (double2*)x_out, results, L, st);
}
