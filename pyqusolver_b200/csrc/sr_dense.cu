// Dense stochastic reconfiguration: the SR matrix S = O_c^H diag(p) O_c / Ns formed on the
// 5th-generation tensor cores, then (S + shift) x = F solved by a float64 blocked Cholesky
// factorisation.  Replaces TDVP's formed-matrix path (QES/NQS/src/tdvp.py:340,433,455: the
// covariance of get_tdvp_standard :1113-1117, solved by the linear solver of _solve_choice
// :1290-1344 with sr_form_matrix=True).
//
//   1. conj(O-bar) and F: float64 sums over the samples of conj(O_s) g_s (one thread per parameter,
//      the structured O_s = [sigma_s, t_s, sigma_s (x) t_s] evaluated on the fly).
//   2. X^T (the centred, weighted O as real rows: Re and Im parts of every complex parameter) as
//      BF16 hi/lo core-matrix tiles, K-major over the samples.
//   3. G = X^T X on tcgen05: one CTA per 128 x 128 tile of the upper triangle, K (samples) streamed
//      through a 3-stage bulk-copy pipeline, hi*hi + hi*lo + lo*hi MMAs into an FP32 TMEM
//      accumulator (the lo*lo term is below 2^-16 relative).
//   4. S from G in float64 (S_re = G_rr + G_ii, S_im = G_ri - G_ir, / Ns), full Hermitian.
//   5. A = S + shift, L L^H = A by 64-column blocks (diagonal block in one CTA, panel triangular
//      solve, register-tiled trailing update of the lower triangle), L y = F, L^H x = y.
//
// Every mbarrier wait is bounded; a time-out sets QES_ERR_TIMEOUT in the status word, the kernel
// still waits (bounded) for its own MMAs, frees its TMEM and returns.
#include "common.cuh"

#include <cuda_bf16.h>
#include "umma.cuh"

#include <algorithm>
#include <cmath>

#define QES_ARG_CHECK(cond, msg) do { if (!(cond)) { qes_set_last_message(msg); return QES_ERR_ARG; } } while (0)

namespace {

constexpr uint32_t kDenseWait = 1u << 22;      // try_wait polls before giving up
constexpr int GR = 128;                        // Gram tile rows / columns
constexpr int GK = 64;                         // samples per K chunk
constexpr int GSTAGES = 3;
constexpr int G_THREADS = 256;                 // warp 0: producer, warp 1: MMA; all 8 warps: epilogue
constexpr int CB = 64;                         // Cholesky block

template <class V> struct DenseT;
template <> struct DenseT<double> { using T = float; static constexpr bool cplx = false; };
template <> struct DenseT<double2> { using T = float2; static constexpr bool cplx = true; };

__device__ __forceinline__ double d_re(double v) { return v; }
__device__ __forceinline__ double d_re(double2 v) { return v.x; }
__device__ __forceinline__ double d_im(double) { return 0.0; }
__device__ __forceinline__ double d_im(double2 v) { return v.y; }
__device__ __forceinline__ double zconj(double v) { return v; }
__device__ __forceinline__ double2 zconj(double2 v) { return make_double2(v.x, -v.y); }
__device__ __forceinline__ double zmul(double a, double b) { return a * b; }
__device__ __forceinline__ double2 zmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double zadd(double a, double b) { return a + b; }
__device__ __forceinline__ double2 zadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double zsub(double a, double b) { return a - b; }
__device__ __forceinline__ double2 zsub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double zscale(double s, double a) { return s * a; }
__device__ __forceinline__ double2 zscale(double s, double2 a) { return make_double2(s * a.x, s * a.y); }
// a - b * conj(c)
__device__ __forceinline__ double zmsc(double a, double b, double c) { return fma(-b, c, a); }
__device__ __forceinline__ double2 zmsc(double2 a, double2 b, double2 c) {
  return make_double2(a.x - (b.x * c.x + b.y * c.y), a.y - (b.y * c.x - b.x * c.y));
}
__device__ __forceinline__ double zfrom(double x, double) { return x; }
__device__ __forceinline__ double2 zfrom(double x, double2) { return make_double2(x, 0.0); }
__device__ __forceinline__ double zzero(double) { return 0.0; }
__device__ __forceinline__ double2 zzero(double2) { return make_double2(0.0, 0.0); }
__device__ __forceinline__ double t_to_d(float t, double) { return (double)t; }
__device__ __forceinline__ double2 t_to_d(float2 t, double2) { return make_double2(t.x, t.y); }

__device__ __forceinline__ uint16_t bf16_bits(float x) { return __bfloat16_as_ushort(__float2bfloat16_rn(x)); }
__device__ __forceinline__ float bf16_val(uint16_t b) { return __bfloat162float(__ushort_as_bfloat16(b)); }
__device__ __forceinline__ uint32_t pack2(uint16_t a, uint16_t b) { return (uint32_t)a | ((uint32_t)b << 16); }

__device__ __forceinline__ void record_error(int* status, int code) {
  if (status) atomicCAS(status, 0, code);
}

// O_sp of parameter p for sample s ([a (ns), b (nh), W (ns x nh)]), as a float64 scalar
template <class V>
__device__ __forceinline__ V o_elem(int ns, int nh, int64_t p, const uint32_t* w_bits, const typename DenseT<V>::T* trow) {
  if (p < ns) return zfrom(((w_bits[p >> 5] >> (p & 31)) & 1u) ? 1.0 : -1.0, V());
  if (p < ns + nh) return t_to_d(trow[p - ns], V());
  const int64_t q = p - ns - nh;
  const int i = (int)(q / nh), j = (int)(q % nh);
  const double sg = ((w_bits[i >> 5] >> (i & 31)) & 1u) ? 1.0 : -1.0;
  return zscale(sg, t_to_d(trow[j], V()));
}

}  // namespace

// out_p = sum_s conj(O_sp) g_s  (float64; one thread per parameter, samples in a fixed order).
// With g_s = p_s / Ns it is conj(O-bar); with g_s = p_s (E_s - <E>) / Ns it is the force F.
template <class V>
__global__ void __launch_bounds__(256) dense_ohg_kernel(int ns, int nh, int64_t n_samples,
                                                         const uint32_t* __restrict__ bits,
                                                         const typename DenseT<V>::T* __restrict__ tt,
                                                         const double2* __restrict__ g, V* __restrict__ out) {
  const int64_t P = (int64_t)ns + nh + (int64_t)ns * nh;
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P) return;
  const int nw = n_words(ns);
  V acc = zzero(V());
  for (int64_t s = 0; s < n_samples; ++s) {
    const V o = o_elem<V>(ns, nh, p, bits + s * nw, tt + s * nh);
    const double2 gs = g[s];
    if constexpr (DenseT<V>::cplx) {
      acc = zadd(acc, zmul(zconj(o), make_double2(gs.x, gs.y)));
    } else {
      acc = acc + o * gs.x;
    }
  }
  out[p] = acc;
}

// X^T as BF16 hi/lo core-matrix tiles: row r of the real embedding (r < P: Re O_c[:, r]; complex:
// P <= r < 2P: Im O_c[:, r - P]) times sqrt(p_s), samples along K.  Tile (row block b, K chunk c)
// at byte ((b * nK + c) * 2 + term) * GR * GK * 2, element offset umma::kmajor_offset(r % GR, k % GK, GR).
template <class V>
__global__ void dense_x_tiles_kernel(int ns, int nh, int64_t n_samples, int rows, int n_rb, int nK,
                                     const uint32_t* __restrict__ bits, const typename DenseT<V>::T* __restrict__ tt,
                                     const float* __restrict__ wts, const V* __restrict__ obar_conj,
                                     uint16_t* __restrict__ out) {
  const int64_t P = (int64_t)ns + nh + (int64_t)ns * nh;
  const int nw = n_words(ns);
  const size_t tile_bytes = (size_t)GR * GK * 2;
  const int64_t items = (int64_t)n_rb * nK * GR * (GK / 8);
  for (int64_t it = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; it < items; it += (int64_t)gridDim.x * blockDim.x) {
    const int r = (int)(it % GR);                       // row within the block (consecutive 16-byte stores)
    const int k8 = (int)((it / GR) % (GK / 8));
    const int64_t bc = it / ((int64_t)GR * (GK / 8));
    const int c = (int)(bc % nK), b = (int)(bc / nK);
    const int64_t row = (int64_t)b * GR + r;
    const bool im = DenseT<V>::cplx && row >= P;
    const int64_t p = im ? row - P : row;
    uint32_t h[4], l[4];
#pragma unroll
    for (int q2 = 0; q2 < 4; ++q2) {
      uint16_t hh[2], ll[2];
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int64_t s = (int64_t)c * GK + 8 * k8 + 2 * q2 + e;
        float x = 0.f;
        if (row < rows && s < n_samples) {
          const V o = zsub(o_elem<V>(ns, nh, p, bits + s * nw, tt + s * nh), zconj(obar_conj[p]));
          const double sw = wts ? sqrt((double)wts[s]) : 1.0;
          x = (float)(sw * (im ? d_im(o) : d_re(o)));
        }
        hh[e] = bf16_bits(x);
        ll[e] = bf16_bits(x - bf16_val(hh[e]));
      }
      h[q2] = pack2(hh[0], hh[1]);
      l[q2] = pack2(ll[0], ll[1]);
    }
    uint8_t* base = reinterpret_cast<uint8_t*>(out) + (((size_t)b * nK + c) * 2) * tile_bytes;
    const uint32_t off = umma::kmajor_offset((uint32_t)r, (uint32_t)(8 * k8), GR);
    *reinterpret_cast<uint4*>(base + off) = make_uint4(h[0], h[1], h[2], h[3]);
    *reinterpret_cast<uint4*>(base + tile_bytes + off) = make_uint4(l[0], l[1], l[2], l[3]);
  }
}

// G tile (I, J), I <= J, of X^T X: D (128 x 128, FP32 in TMEM) += A_I hi B_J hi + A_I hi B_J lo +
// A_I lo B_J hi over the K chunks.  Warp 0 lane 0 issues the bulk copies, warp 1 lane 0 the MMAs;
// after the last commit every warp reads its TMEM lane quarter (warps w and w + 4 split the columns)
// and writes the tile row-major into G (ldg = padded row count).
__global__ void __launch_bounds__(G_THREADS, 1) dense_gram_kernel(int n_rb, int nK, const uint16_t* __restrict__ xt,
                                                                  float* __restrict__ G, int64_t ldg,
                                                                  int* __restrict__ status) {
  extern __shared__ __align__(128) uint8_t smem[];
  constexpr uint32_t term = GR * GK * 2;                    // one 128 x 64 BF16 tile: 16 KB
  constexpr uint32_t stage_bytes = 4 * term;                // A hi, A lo, B hi, B lo
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + GSTAGES * stage_bytes);
  uint64_t* empty = full + GSTAGES;
  uint64_t* done = empty + GSTAGES;
  uint32_t* tslot = reinterpret_cast<uint32_t*>(done + 1);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  // tile index -> (I, J) with I <= J: row I holds n_rb - I tiles
  int I = 0;
  int64_t t = blockIdx.x;
  while (I < n_rb && t >= n_rb - I) { t -= n_rb - I; ++I; }
  const int J = I + (int)t;
  const uint8_t* ga = reinterpret_cast<const uint8_t*>(xt) + (size_t)I * nK * 2 * term;
  const uint8_t* gb = reinterpret_cast<const uint8_t*>(xt) + (size_t)J * nK * 2 * term;
  if (tid == 0) {
    for (int q = 0; q < GSTAGES; ++q) {
      umma::mbar_init(&full[q], 1);
      umma::mbar_init(&empty[q], 1);
    }
    umma::mbar_init(done, 1);
    umma::fence_mbar_init();
  }
  if (warp == 0) {
    umma::tmem_alloc(tslot, GR);
    umma::tmem_relinquish();
  }
  umma::tc_fence_before();
  __syncthreads();
  umma::tc_fence_after();
  const uint32_t tbase = *tslot;
  if (warp == 0 && lane == 0) {
    // producer: chunk c into stage c % GSTAGES once the MMAs of chunk c - GSTAGES have completed
    for (int c = 0; c < nK; ++c) {
      const int s = c % GSTAGES;
      if (c >= GSTAGES && !umma::mbar_wait(&empty[s], ((c / GSTAGES) - 1) & 1, kDenseWait)) {
        record_error(status, QES_ERR_TIMEOUT);
        break;
      }
      uint8_t* st = smem + s * stage_bytes;
      umma::mbar_arrive_expect_tx(&full[s], stage_bytes);
      umma::bulk_g2s(st, ga + (size_t)c * 2 * term, 2 * term, &full[s]);
      umma::bulk_g2s(st + 2 * term, gb + (size_t)c * 2 * term, 2 * term, &full[s]);
    }
  } else if (warp == 1 && lane == 0) {
    const uint32_t idesc = umma::idesc_bf16_f32(GR, GR);
    int c = 0;
    for (; c < nK; ++c) {
      const int s = c % GSTAGES;
      if (!umma::mbar_wait(&full[s], (c / GSTAGES) & 1, kDenseWait)) {
        record_error(status, QES_ERR_TIMEOUT);
        break;
      }
      umma::tc_fence_after();
      const uint32_t sa = umma::smem_u32(smem + s * stage_bytes);
      const uint32_t ahi = sa, alo = sa + term, bhi = sa + 2 * term, blo = sa + 3 * term;
      for (int kk = 0; kk < GK / 16; ++kk) {
        const uint32_t ko = 2u * kk * GR * 16u;
        const uint64_t dah = umma::smem_desc(ahi + ko, GR * 16u, 128u);
        const uint64_t dal = umma::smem_desc(alo + ko, GR * 16u, 128u);
        const uint64_t dbh = umma::smem_desc(bhi + ko, GR * 16u, 128u);
        const uint64_t dbl = umma::smem_desc(blo + ko, GR * 16u, 128u);
        umma::mma_bf16(tbase, dah, dbh, idesc, (c > 0 || kk > 0) ? 1u : 0u);
        umma::mma_bf16(tbase, dah, dbl, idesc, 1u);
        umma::mma_bf16(tbase, dal, dbh, idesc, 1u);
      }
      umma::mma_commit(&empty[s]);
    }
    umma::mma_commit(done);            // arrives once every MMA issued above has completed
  }
  __syncthreads();
  if (!umma::mbar_wait(done, 0, kDenseWait)) record_error(status, QES_ERR_TIMEOUT);
  umma::tc_fence_after();
  // epilogue: warp w reads lanes 32 (w % 4) .. + 31 (tile rows), column half w / 4
  const int quarter = warp & 3, half = warp >> 2;
  const int rloc = 32 * quarter + lane;
  const uint32_t lane_addr = tbase + ((uint32_t)(32 * quarter) << 16);
  float* grow = G + ((int64_t)I * GR + rloc) * ldg + (int64_t)J * GR;
  for (int c16 = half * 4; c16 < half * 4 + 4; ++c16) {
    float v[16];
    umma::tmem_ld16(lane_addr + 16 * c16, v);
#pragma unroll
    for (int q = 0; q < 16; q += 4)
      *reinterpret_cast<float4*>(grow + 16 * c16 + q) = make_float4(v[q], v[q + 1], v[q + 2], v[q + 3]);
  }
  umma::tc_fence_before();
  __syncthreads();
  if (warp == 0) umma::tmem_dealloc(tbase, GR);
}

// g vectors of one solve (one block): gw_s = p_s / Ns (-> conj(O-bar)), ge_s = p_s (E_s - <E>) / Ns
// (-> F), with <E> = sum p E / Ns written to emean[0..1]; eloc == nullptr (the Gram-only call): gw only
__global__ void __launch_bounds__(1024) dense_g_kernel(int64_t n, const float2* __restrict__ eloc,
                                                        const float* __restrict__ wts, double2* __restrict__ gw,
                                                        double2* __restrict__ ge, double* __restrict__ emean) {
  __shared__ double rr[32], ri[32];
  __shared__ double m[2];
  double sr = 0.0, si = 0.0;
  for (int64_t s = threadIdx.x; eloc && s < n; s += blockDim.x) {      // no E_loc in the Gram-only call
    const double f = wts ? (double)wts[s] : 1.0;
    sr += f * eloc[s].x;
    si += f * eloc[s].y;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    sr += __shfl_xor_sync(0xffffffffu, sr, o);
    si += __shfl_xor_sync(0xffffffffu, si, o);
  }
  if ((threadIdx.x & 31) == 0) { rr[threadIdx.x >> 5] = sr; ri[threadIdx.x >> 5] = si; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0.0, b = 0.0;
    for (int q = 0; q < (int)(blockDim.x >> 5); ++q) { a += rr[q]; b += ri[q]; }
    m[0] = a / (double)n;
    m[1] = b / (double)n;
    if (emean) { emean[0] = m[0]; emean[1] = m[1]; }
  }
  __syncthreads();
  const double inv = 1.0 / (double)n;
  for (int64_t s = threadIdx.x; s < n; s += blockDim.x) {
    const double f = (wts ? (double)wts[s] : 1.0) * inv;
    gw[s] = make_double2(f, 0.0);
    if (ge) ge[s] = make_double2(f * (eloc[s].x - m[0]), f * (eloc[s].y - m[1]));
  }
}

// A = S + shift I with S from the Gram tiles (float64, full Hermitian, row-major P x P):
// complex S_pq = (G[p][q] + G[P+p][P+q] + i (G[p][P+q] - G[P+p][q])) / Ns, real S_pq = G[p][q] / Ns.
// Only the tiles (I <= J) of G were formed; every element is read from the upper triangle
// (a <= b; the mirror below it), so S comes out exactly Hermitian.
template <class V>
__global__ void dense_combine_kernel(int64_t P, int64_t ldg, const float* __restrict__ G, double inv_n,
                                     double shift, V* __restrict__ A) {
  auto g = [&](int64_t a, int64_t b) -> double { return (double)((a <= b) ? G[a * ldg + b] : G[b * ldg + a]); };
  const int64_t total = P * P;
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int64_t p = idx / P, q = idx % P;
    V v;
    if constexpr (DenseT<V>::cplx) {
      v = make_double2((g(p, q) + g(P + p, P + q)) * inv_n, (g(p, P + q) - g(P + p, q)) * inv_n);
      if (p == q) v.x += shift;
    } else {
      v = g(p, q) * inv_n;
      if (p == q) v += shift;
    }
    A[idx] = v;
  }
}

// ---------------------------------------------------------------- Cholesky (lower, row-major, lda = P)
// diagonal block [k0, k0 + nb): unblocked right-looking factorisation in shared memory.  A pivot that
// is not positive (S + shift not positive definite in float64) sets *info = column + 1 and is
// replaced by 1 so that the factorisation finishes without NaN; the host reports the failure.
template <class V>
__global__ void __launch_bounds__(256) chol_diag_kernel(V* __restrict__ A, int64_t lda, int64_t k0, int nb,
                                                        int* __restrict__ info) {
  extern __shared__ __align__(16) uint8_t csm[];
  V* L = reinterpret_cast<V*>(csm);                         // [nb][nb + 1]
  const int ld = nb + 1;
  for (int e = threadIdx.x; e < nb * nb; e += blockDim.x) {
    const int i = e / nb, j = e % nb;
    L[i * ld + j] = (j <= i) ? A[(k0 + i) * lda + k0 + j] : zzero(V());
  }
  __syncthreads();
  for (int j = 0; j < nb; ++j) {
    if (threadIdx.x == 0) {
      double d = d_re(L[j * ld + j]);
      if (!(d > 0.0)) {
        atomicCAS(info, 0, (int)(k0 + j + 1));
        d = 1.0;
      }
      L[j * ld + j] = zfrom(sqrt(d), V());
    }
    __syncthreads();
    const double inv = 1.0 / d_re(L[j * ld + j]);
    for (int i = j + 1 + threadIdx.x; i < nb; i += blockDim.x) L[i * ld + j] = zscale(inv, L[i * ld + j]);
    __syncthreads();
    // trailing update of the lower triangle: L[i][k] -= L[i][j] conj(L[k][j]), j < k <= i
    const int m = nb - j - 1;
    for (int e = threadIdx.x; e < m * m; e += blockDim.x) {
      const int i = j + 1 + e / m, k = j + 1 + e % m;
      if (k <= i) L[i * ld + k] = zmsc(L[i * ld + k], L[i * ld + j], L[k * ld + j]);
    }
    __syncthreads();
  }
  for (int e = threadIdx.x; e < nb * nb; e += blockDim.x) {
    const int i = e / nb, j = e % nb;
    if (j <= i) A[(k0 + i) * lda + k0 + j] = L[i * ld + j];
  }
}

// panel below the diagonal block: row x of A[k0 + nb .. P)[k0 .. k0 + nb) becomes x L_kk^{-H}
// (forward substitution over the block's columns, one thread per row, L_kk in shared memory)
template <class V>
__global__ void __launch_bounds__(128) chol_panel_kernel(V* __restrict__ A, int64_t lda, int64_t k0, int nb, int64_t P) {
  extern __shared__ __align__(16) uint8_t csm[];
  V* L = reinterpret_cast<V*>(csm);                         // [nb][nb]
  for (int e = threadIdx.x; e < nb * nb; e += blockDim.x) {
    const int i = e / nb, j = e % nb;
    L[e] = (j <= i) ? A[(k0 + i) * lda + k0 + j] : zzero(V());
  }
  __syncthreads();
  const int64_t row = k0 + nb + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= P) return;
  V* x = A + row * lda + k0;
  for (int j = 0; j < nb; ++j) {
    V a = x[j];
    for (int l = 0; l < j; ++l) a = zmsc(a, x[l], L[j * nb + l]);
    x[j] = zscale(1.0 / d_re(L[j * nb + j]), a);
  }
}

// trailing update of the lower triangle: A[I][J] -= L[I][K] L[J][K]^H for the 64 x 64 tiles I >= J
// of rows / columns [k1, P), K = [k0, k0 + nb); 16 x 16 threads with 4 x 4 register tiles
template <class V>
__global__ void __launch_bounds__(256) chol_update_kernel(V* __restrict__ A, int64_t lda, int64_t k0, int nb,
                                                          int64_t k1, int64_t P) {
  constexpr int TK = 16;
  __shared__ V Li[CB][TK + 1];
  __shared__ V Lj[CB][TK + 1];
  const int bi = blockIdx.y, bj = blockIdx.x;
  if (bj > bi) return;
  const int64_t i0 = k1 + (int64_t)bi * CB, j0 = k1 + (int64_t)bj * CB;
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  V acc[4][4];
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int c = 0; c < 4; ++c) acc[r][c] = zzero(V());
  for (int kk = 0; kk < nb; kk += TK) {
    __syncthreads();
    for (int e = threadIdx.x; e < CB * TK; e += 256) {
      const int r = e / TK, k = e % TK;
      const int64_t gi = i0 + r, gj = j0 + r;
      const bool kin = kk + k < nb;
      Li[r][k] = (gi < P && kin) ? A[gi * lda + k0 + kk + k] : zzero(V());
      Lj[r][k] = (gj < P && kin) ? A[gj * lda + k0 + kk + k] : zzero(V());
    }
    __syncthreads();
#pragma unroll 4
    for (int k = 0; k < TK; ++k) {
      V a[4], b[4];
#pragma unroll
      for (int r = 0; r < 4; ++r) a[r] = Li[ty + 16 * r][k];
#pragma unroll
      for (int c = 0; c < 4; ++c) b[c] = zconj(Lj[tx + 16 * c][k]);
#pragma unroll
      for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int c = 0; c < 4; ++c) acc[r][c] = zadd(acc[r][c], zmul(a[r], b[c]));
    }
  }
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    const int64_t gi = i0 + ty + 16 * r;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const int64_t gj = j0 + tx + 16 * c;
      if (gi < P && gj <= gi) A[gi * lda + gj] = zsub(A[gi * lda + gj], acc[r][c]);
    }
  }
}

namespace {
__device__ __forceinline__ double dwarp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double2 dwarp_sum(double2 v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
    v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
  }
  return v;
}
}  // namespace

// ---------------------------------------------------------------- triangular solves with L (row-major)
// L y = b on the diagonal block [k0, k0 + nb) (one warp; lanes split the dot products)
template <class V>
__global__ void trsv_fwd_diag_kernel(const V* __restrict__ A, int64_t lda, int64_t k0, int nb, V* __restrict__ y) {
  const int lane = threadIdx.x;
  for (int j = 0; j < nb; ++j) {
    V part = zzero(V());
    for (int l = lane; l < j; l += 32) part = zadd(part, zmul(A[(k0 + j) * lda + k0 + l], y[k0 + l]));
    part = dwarp_sum(part);
    if (lane == 0) y[k0 + j] = zscale(1.0 / d_re(A[(k0 + j) * lda + k0 + j]), zsub(y[k0 + j], part));
    __syncwarp();
  }
}
// y_i -= sum_{l in block} L_il y_l for the rows below the block (one warp per row)
template <class V>
__global__ void trsv_fwd_update_kernel(const V* __restrict__ A, int64_t lda, int64_t k0, int nb, int64_t P,
                                       V* __restrict__ y) {
  const int lane = threadIdx.x & 31;
  const int64_t i = k0 + nb + (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (i >= P) return;
  V part = zzero(V());
  for (int l = lane; l < nb; l += 32) part = zadd(part, zmul(A[i * lda + k0 + l], y[k0 + l]));
  part = dwarp_sum(part);
  if (lane == 0) y[i] = zsub(y[i], part);
}
// L^H x = y on the diagonal block, j descending: x_j = (y_j - sum_{l > j} conj(L_lj) x_l) / L_jj
template <class V>
__global__ void trsv_bwd_diag_kernel(const V* __restrict__ A, int64_t lda, int64_t k0, int nb, V* __restrict__ y) {
  const int lane = threadIdx.x;
  for (int j = nb - 1; j >= 0; --j) {
    V part = zzero(V());
    for (int l = j + 1 + lane; l < nb; l += 32) part = zadd(part, zmul(zconj(A[(k0 + l) * lda + k0 + j]), y[k0 + l]));
    part = dwarp_sum(part);
    if (lane == 0) y[k0 + j] = zscale(1.0 / d_re(A[(k0 + j) * lda + k0 + j]), zsub(y[k0 + j], part));
    __syncwarp();
  }
}
// y_i -= sum_{l in block} conj(L_li) x_l for the rows above the block (one thread per row: the reads
// L[l][i] are consecutive across the threads)
template <class V>
__global__ void trsv_bwd_update_kernel(const V* __restrict__ A, int64_t lda, int64_t k0, int nb, V* __restrict__ y) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= k0) return;
  V part = zzero(V());
  for (int l = 0; l < nb; ++l) part = zadd(part, zmul(zconj(A[(k0 + l) * lda + i]), y[k0 + l]));
  y[i] = zsub(y[i], part);
}

// per-row |b - M x|^2 and |b|^2 of the dense system (one warp per row), then one block sums them
template <class V>
__global__ void dense_resid_kernel(const V* __restrict__ M, int64_t P, const V* __restrict__ x,
                                   const V* __restrict__ b, double* __restrict__ rr, double* __restrict__ bb) {
  const int lane = threadIdx.x & 31;
  const int64_t i = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (i >= P) return;
  V part = zzero(V());
  for (int64_t q = lane; q < P; q += 32) part = zadd(part, zmul(M[i * P + q], x[q]));
  part = dwarp_sum(part);
  if (lane == 0) {
    const V r = zsub(b[i], part);
    rr[i] = d_re(r) * d_re(r) + d_im(r) * d_im(r);
    bb[i] = d_re(b[i]) * d_re(b[i]) + d_im(b[i]) * d_im(b[i]);
  }
}
__global__ void __launch_bounds__(1024) dense_sum2_kernel(int64_t n, const double* __restrict__ a,
                                                           const double* __restrict__ b, double* __restrict__ out) {
  __shared__ double ra[32], rb[32];
  double sa = 0.0, sb = 0.0;
  for (int64_t k = threadIdx.x; k < n; k += blockDim.x) { sa += a[k]; sb += b[k]; }
  sa = dwarp_sum(sa);
  sb = dwarp_sum(sb);
  if ((threadIdx.x & 31) == 0) { ra[threadIdx.x >> 5] = sa; rb[threadIdx.x >> 5] = sb; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double x = 0.0, y = 0.0;
    for (int q = 0; q < (int)(blockDim.x >> 5); ++q) { x += ra[q]; y += rb[q]; }
    out[0] = x;
    out[1] = y;
  }
}
template <class V>
__global__ void dense_scale_copy_kernel(int64_t n, double s, const V* __restrict__ x, V* __restrict__ out) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x)
    out[k] = zscale(s, x[k]);
}

// ================================================================================================
// host side
// ================================================================================================
namespace {

struct DenseWork {
  int64_t P = 0, rows = 0;
  int n_rb = 0, nK = 0;
  double2 *gw = nullptr, *ge = nullptr;
  double* emean = nullptr;      // [2]
  void *obar = nullptr, *F = nullptr, *y = nullptr;     // [P] of V
  uint16_t* xt = nullptr;       // X^T tiles
  float* G = nullptr;           // [Rp][Rp]; reused as the copy of A for the residual
  void* A = nullptr;            // [P][P] of V (solve only; the caller's S in the Gram-only call)
  double *rr = nullptr, *bb = nullptr, *scal = nullptr;
  int* flags = nullptr;         // [0] Cholesky info, [1] tensor-core status
  size_t total = 0;
};

size_t al256(size_t x) { return (x + 255) & ~(size_t)255; }

// with_A: the factorisation buffer (solve); without, the Gram-only call writes S into the caller's array
DenseWork dense_layout(int dtype, int ns, int nh, int64_t n, bool with_A, char* base) {
  DenseWork W;
  const bool cplx = dtype == QES_DTYPE_C64;
  const size_t vs = cplx ? sizeof(double2) : sizeof(double);
  W.P = (int64_t)ns + nh + (int64_t)ns * nh;
  W.rows = cplx ? 2 * W.P : W.P;
  W.n_rb = (int)((W.rows + GR - 1) / GR);
  W.nK = (int)((n + GK - 1) / GK);
  const int64_t Rp = (int64_t)W.n_rb * GR;
  size_t off = 0;
  auto take = [&](size_t bytes) { char* p = base ? base + off : nullptr; off += al256(bytes); return p; };
  W.gw = (double2*)take((size_t)n * sizeof(double2));
  W.ge = (double2*)take((size_t)n * sizeof(double2));
  W.emean = (double*)take(4 * sizeof(double));
  W.obar = take((size_t)W.P * vs);
  W.F = take((size_t)W.P * vs);
  W.y = take((size_t)W.P * vs);
  W.xt = (uint16_t*)take((size_t)W.n_rb * W.nK * 2 * GR * GK * 2);
  W.G = (float*)take(std::max((size_t)Rp * Rp * sizeof(float), with_A ? (size_t)W.P * W.P * vs : 0));
  W.A = with_A ? take((size_t)W.P * W.P * vs) : nullptr;
  W.rr = (double*)take((size_t)W.P * sizeof(double));
  W.bb = (double*)take((size_t)W.P * sizeof(double));
  W.scal = (double*)take(8 * sizeof(double));
  W.flags = (int*)take(8 * sizeof(int));
  W.total = off;
  return W;
}

constexpr size_t kDenseMaxBytes = (size_t)100 << 30;     // the dense path refuses larger systems

template <class V>
int dense_gram_t(int ns, int nh, int64_t n, const uint32_t* bits, const typename DenseT<V>::T* tt,
                 const float2* eloc, const float* probs, double shift, V* A, const DenseWork& W, cudaStream_t st) {
  QES_CUDA_CHECK(cudaMemsetAsync(W.flags, 0, 8 * sizeof(int), st));
  dense_g_kernel<<<1, 1024, 0, st>>>(n, eloc, probs, W.gw, eloc ? W.ge : nullptr, W.emean);
  const int pb = (int)((W.P + 255) / 256);
  dense_ohg_kernel<V><<<pb, 256, 0, st>>>(ns, nh, n, bits, tt, W.gw, (V*)W.obar);
  const int64_t items = (int64_t)W.n_rb * W.nK * GR * (GK / 8);
  dense_x_tiles_kernel<V><<<(unsigned)std::min<int64_t>((items + 255) / 256, 4 * 1184), 256, 0, st>>>(
      ns, nh, n, (int)W.rows, W.n_rb, W.nK, bits, tt, probs, (const V*)W.obar, W.xt);
  QES_LAUNCH_CHECK_N(3);
  const size_t smem = (size_t)GSTAGES * 4 * GR * GK * 2 + 8 * (2 * GSTAGES + 1) + 16;
  QES_CUDA_CHECK(cudaFuncSetAttribute(dense_gram_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int64_t tiles = (int64_t)W.n_rb * (W.n_rb + 1) / 2;
  QES_ARG_CHECK(tiles < (1ll << 31), "dense SR: too many Gram tiles");
  const int pf = qes_prof_begin(QES_PROF_GRAM, st);
  dense_gram_kernel<<<(unsigned)tiles, G_THREADS, smem, st>>>(W.n_rb, W.nK, W.xt, W.G, (int64_t)W.n_rb * GR,
                                                              W.flags + 1);
  QES_LAUNCH_CHECK();
  qes_prof_end(pf, st);
  const int64_t tot = W.P * W.P;
  dense_combine_kernel<V><<<(unsigned)std::min<int64_t>((tot + 255) / 256, 8 * 1184), 256, 0, st>>>(
      W.P, (int64_t)W.n_rb * GR, W.G, 1.0 / (double)n, shift, A);
  QES_LAUNCH_CHECK();
  return QES_OK;
}

int dense_read_flags(const DenseWork& W, cudaStream_t st, int* info) {
  int h[2] = {0, 0};
  QES_CUDA_CHECK(cudaMemcpyAsync(h, W.flags, 2 * sizeof(int), cudaMemcpyDeviceToHost, st));
  QES_CUDA_CHECK(cudaStreamSynchronize(st));
  if (h[1] != 0) {
    qes_set_last_message("dense SR: a bounded tensor-core wait gave up");
    return QES_ERR_TIMEOUT;
  }
  if (info) *info = h[0];
  return QES_OK;
}

template <class V>
int dense_solve_t(int ns, int nh, int64_t n, const uint32_t* bits, const typename DenseT<V>::T* tt,
                  const float2* eloc, const float* probs, const qes_sr_options* opt, V* x_out, qes_sr_result* res,
                  const DenseWork& W, cudaStream_t st) {
  const int64_t P = W.P;
  V* A = (V*)W.A;
  V* y = (V*)W.y;
  int rc = dense_gram_t<V>(ns, nh, n, bits, tt, eloc, probs, opt->shift, A, W, st);
  if (rc) return rc;
  // keep S + shift for the residual check (the Gram tiles are no longer needed)
  QES_CUDA_CHECK(cudaMemcpyAsync(W.G, A, (size_t)P * P * sizeof(V), cudaMemcpyDeviceToDevice, st));
  const int pb = (int)((P + 255) / 256);
  dense_ohg_kernel<V><<<pb, 256, 0, st>>>(ns, nh, n, bits, tt, W.ge, (V*)W.F);
  QES_LAUNCH_CHECK();
  // blocked Cholesky
  const size_t sm_diag = (size_t)CB * (CB + 1) * sizeof(V), sm_panel = (size_t)CB * CB * sizeof(V);
  QES_CUDA_CHECK(cudaFuncSetAttribute(chol_diag_kernel<V>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_diag));
  QES_CUDA_CHECK(cudaFuncSetAttribute(chol_panel_kernel<V>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)sm_panel));
  const int pfc = qes_prof_begin(QES_PROF_CHOL, st);
  for (int64_t k0 = 0; k0 < P; k0 += CB) {
    const int nb = (int)std::min<int64_t>(CB, P - k0);
    chol_diag_kernel<V><<<1, 256, sm_diag, st>>>(A, P, k0, nb, W.flags);
    const int64_t k1 = k0 + nb, rest = P - k1;
    if (rest > 0) {
      chol_panel_kernel<V><<<(unsigned)((rest + 127) / 128), 128, sm_panel, st>>>(A, P, k0, nb, P);
      const unsigned nt = (unsigned)((rest + CB - 1) / CB);
      chol_update_kernel<V><<<dim3(nt, nt), 256, 0, st>>>(A, P, k0, nb, k1, P);
      QES_LAUNCH_CHECK_N(3);
    } else {
      QES_LAUNCH_CHECK();
    }
  }
  qes_prof_end(pfc, st);
  // L y = F, L^H x = y
  QES_CUDA_CHECK(cudaMemcpyAsync(y, W.F, (size_t)P * sizeof(V), cudaMemcpyDeviceToDevice, st));
  for (int64_t k0 = 0; k0 < P; k0 += CB) {
    const int nb = (int)std::min<int64_t>(CB, P - k0);
    trsv_fwd_diag_kernel<V><<<1, 32, 0, st>>>(A, P, k0, nb, y);
    const int64_t rest = P - k0 - nb;
    if (rest > 0) trsv_fwd_update_kernel<V><<<(unsigned)((rest + 7) / 8), 256, 0, st>>>(A, P, k0, nb, P, y);
  }
  for (int64_t k0 = ((P - 1) / CB) * CB; k0 >= 0; k0 -= CB) {
    const int nb = (int)std::min<int64_t>(CB, P - k0);
    trsv_bwd_diag_kernel<V><<<1, 32, 0, st>>>(A, P, k0, nb, y);
    if (k0 > 0) trsv_bwd_update_kernel<V><<<(unsigned)((k0 + 255) / 256), 256, 0, st>>>(A, P, k0, nb, y);
  }
  QES_LAUNCH_CHECK();
  // residual in S + shift (kept in W.G), then x_out = rhs_prefactor * x
  dense_resid_kernel<V><<<(unsigned)((P + 7) / 8), 256, 0, st>>>((const V*)W.G, P, y, (const V*)W.F, W.rr, W.bb);
  dense_sum2_kernel<<<1, 1024, 0, st>>>(P, W.rr, W.bb, W.scal);
  dense_scale_copy_kernel<V><<<(unsigned)std::min<int64_t>((P + 255) / 256, 1184), 256, 0, st>>>(
      P, opt->rhs_prefactor, y, x_out);
  QES_LAUNCH_CHECK_N(3);
  double sc[2] = {0, 0}, em[2] = {0, 0};
  QES_CUDA_CHECK(cudaMemcpyAsync(sc, W.scal, 2 * sizeof(double), cudaMemcpyDeviceToHost, st));
  QES_CUDA_CHECK(cudaMemcpyAsync(em, W.emean, 2 * sizeof(double), cudaMemcpyDeviceToHost, st));
  int info = 0;
  if ((rc = dense_read_flags(W, st, &info))) return rc;
  if (res) {
    res->iterations = 0;
    res->converged = info == 0 ? 1 : 0;
    res->residual = sqrt(sc[0]);
    res->rhs_norm = sqrt(sc[1]);
    res->e_mean_re = em[0];
    res->e_mean_im = em[1];
    res->true_residual = sc[1] > 0.0 ? sqrt(sc[0] / sc[1]) : 0.0;
    res->acond = -1.0;
  }
  if (info != 0) {
    qes_set_last_message("dense SR: S + shift is not positive definite in float64 (Cholesky pivot <= 0)");
    return QES_ERR_NOT_CONVERGED;
  }
  return QES_OK;
}

int dense_check(int dtype, int ns, int nh, int64_t n, bool with_A, void* ws, size_t ws_bytes, DenseWork* W) {
  QES_ARG_CHECK(ns > 0 && nh > 0 && n > 0, "dense SR: bad sizes");
  QES_ARG_CHECK(dtype == QES_DTYPE_F32 || dtype == QES_DTYPE_C64, "dense SR: bad dtype");
  const DenseWork probe = dense_layout(dtype, ns, nh, n, with_A, nullptr);
  if (probe.total > kDenseMaxBytes) {
    qes_set_last_message("dense SR: the formed S matrix and its workspace exceed 100 GB; use the matrix-free solve");
    return QES_ERR_SIZE;
  }
  if (!ws || ws_bytes < probe.total || (reinterpret_cast<uintptr_t>(ws) & 255) != 0) {
    qes_set_last_message("dense SR: workspace too small or not 256-byte aligned");
    return QES_ERR_WORKSPACE;
  }
  *W = dense_layout(dtype, ns, nh, n, with_A, (char*)ws);
  return QES_OK;
}

}  // namespace

extern "C" int qes_sr_dense_workspace_bytes(int dtype, int ns, int nh, int64_t n_samples, int gram_only,
                                            size_t* bytes) {
  QES_ARG_CHECK(bytes && ns > 0 && nh > 0 && n_samples > 0, "qes_sr_dense_workspace_bytes: bad args");
  QES_ARG_CHECK(dtype == QES_DTYPE_F32 || dtype == QES_DTYPE_C64, "qes_sr_dense_workspace_bytes: bad dtype");
  const DenseWork W = dense_layout(dtype, ns, nh, n_samples, gram_only == 0, nullptr);
  *bytes = W.total;
  if (W.total > kDenseMaxBytes) {
    qes_set_last_message("dense SR: the formed S matrix and its workspace exceed 100 GB; use the matrix-free solve");
    return QES_ERR_SIZE;
  }
  return QES_OK;
}

extern "C" int qes_sr_gram(int dtype, int ns, int nh, int64_t n_samples, const uint32_t* bits, const void* tanh_theta,
                           const float* probs, void* s_out, void* workspace, size_t workspace_bytes, void* stream) {
  QES_ARG_CHECK(bits && tanh_theta && s_out, "qes_sr_gram: bad args");
  DenseWork W;
  int rc = dense_check(dtype, ns, nh, n_samples, false, workspace, workspace_bytes, &W);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  if (dtype == QES_DTYPE_C64)
    rc = dense_gram_t<double2>(ns, nh, n_samples, bits, (const float2*)tanh_theta, nullptr, probs, 0.0,
                               (double2*)s_out, W, st);
  else
    rc = dense_gram_t<double>(ns, nh, n_samples, bits, (const float*)tanh_theta, nullptr, probs, 0.0,
                              (double*)s_out, W, st);
  if (rc) return rc;
  return dense_read_flags(W, st, nullptr);
}

extern "C" int qes_sr_solve_dense(int dtype, int ns, int nh, int64_t n_samples, const uint32_t* bits,
                                  const void* tanh_theta, const void* eloc, const float* probs,
                                  const qes_sr_options* opt, void* x_out, qes_sr_result* result, void* workspace,
                                  size_t workspace_bytes, void* stream) {
  QES_ARG_CHECK(bits && tanh_theta && eloc && opt && x_out, "qes_sr_solve_dense: bad args");
  QES_ARG_CHECK(opt->shift >= 0.0, "qes_sr_solve_dense: bad options");
  DenseWork W;
  int rc = dense_check(dtype, ns, nh, n_samples, true, workspace, workspace_bytes, &W);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  if (dtype == QES_DTYPE_C64)
    return dense_solve_t<double2>(ns, nh, n_samples, bits, (const float2*)tanh_theta, (const float2*)eloc, probs, opt,
                                  (double2*)x_out, result, W, st);
  return dense_solve_t<double>(ns, nh, n_samples, bits, (const float*)tanh_theta, (const float2*)eloc, probs, opt,
                               (double*)x_out, result, W, st);
}
