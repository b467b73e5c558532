// RBM forward on the 5th-generation tensor cores: theta = Sigma W + b for a batch of samples.
//
//   D (128 samples x NR units) = Sigma_tile (128 x ns, BF16 +-1, exact) . W^T
// with W split into three BF16 terms (W = W1 + W2 + W3 holds every float32 W exactly), so the
// three MMAs per k-step give Sigma W with float32 accumulation in TMEM.  Complex W has its real
// and imaginary parts as separate operand rows ([Re W | Im W] per N chunk), i.e. two real
// GEMMs.  Hidden units are tiled in N chunks of NC (NR = NC or 2 NC rows <= 512 TMEM columns);
// grid = (sample tiles, N chunks).  K (sites) streams through a bulk-copy pipeline; the epilogue
// adds b, writes tanh(theta) (and theta) and per-chunk partial sums of log cosh(theta), which a
// second kernel adds to sigma . a to give log psi.
//
// Every mbarrier wait is bounded; a time-out sets QES_ERR_TIMEOUT in *status (read by the host).
#include "common.cuh"
#include "umma.cuh"

#include <algorithm>
#include <cuda_bf16.h>

#define QES_ARG_CHECK(cond, msg) do { if (!(cond)) { qes_set_last_message(msg); return QES_ERR_ARG; } } while (0)

namespace {
constexpr uint32_t kWait = 1u << 22;
constexpr int kThr = 512;
constexpr int kWarpsT = kThr / 32;
constexpr int kCG = kWarpsT / 4;
constexpr int kKCH = 32;                 // sites per pipeline stage
constexpr size_t kSmemLimit = 220 * 1024;

__device__ __forceinline__ uint16_t bf(float x) { return __bfloat16_as_ushort(__float2bfloat16_rn(x)); }
__device__ __forceinline__ float bfv(uint16_t b) { return __bfloat162float(__ushort_as_bfloat16(b)); }
__device__ __forceinline__ uint32_t pk2(uint16_t a, uint16_t b) { return (uint32_t)a | ((uint32_t)b << 16); }
__device__ __forceinline__ uint4 pk8(const uint16_t (&v)[8]) {
  return make_uint4(pk2(v[0], v[1]), pk2(v[2], v[3]), pk2(v[4], v[5]), pk2(v[6], v[7]));
}
__device__ __forceinline__ float wre(const float* w, int64_t k) { return w[k]; }
__device__ __forceinline__ float wre(const float2* w, int64_t k) { return w[k].x; }
__device__ __forceinline__ float wim(const float*, int64_t) { return 0.f; }
__device__ __forceinline__ float wim(const float2* w, int64_t k) { return w[k].y; }
}  // namespace

struct ThetaDims {
  int ns, nh, KP, nK;          // sites, hidden units, sites padded to kKCH, K chunks
  int NC, NR, nnc;             // units per N chunk, operand rows per chunk (NC or 2 NC), N chunks
  int n_tiles, stages, smem, tmem_cols;
};

static int pow2_ge(int x) { int p = 32; while (p < x) p <<= 1; return p; }

static bool theta_plan(bool cplx, int ns, int nh, int64_t n, ThetaDims* o) {
  ThetaDims d{};
  d.ns = ns; d.nh = nh;
  d.KP = (ns + kKCH - 1) / kKCH * kKCH;
  d.nK = d.KP / kKCH;
  const int H = cplx ? 2 : 1;
  const int Mp = (nh + 15) / 16 * 16;
  int nc = std::min(Mp, 512 / H / 16 * 16);
  if (nc < 16) return false;
  d.NC = nc;
  d.NR = H * nc;
  d.nnc = (nh + nc - 1) / nc;
  d.n_tiles = (int)((n + 127) / 128);
  const size_t stage = 128u * kKCH * 2 + 3u * (size_t)d.NR * kKCH * 2;
  const size_t extra = 8 * 9 + 16 + 64;
  const int S = (int)std::min<size_t>(4, (kSmemLimit - extra) / stage);
  if (S < 2) return false;
  d.stages = S;
  d.smem = (int)(S * stage + extra);
  d.tmem_cols = pow2_ge(d.NR);
  if (d.tmem_cols > 512) return false;
  *o = d;
  return true;
}

// Sigma rows: tile t, K chunk c -> (t * nK + c) * (128 * kKCH * 2) + kmajor(r, k % kKCH, 128)
__global__ void theta_sig_rows_kernel(ThetaDims d, int64_t n, const uint32_t* __restrict__ bits,
                                      uint16_t* __restrict__ out) {
  const int nw = n_words(d.ns);
  const int64_t items = (int64_t)d.n_tiles * 128 * (d.KP / 8);
  for (int64_t it = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; it < items; it += (int64_t)gridDim.x * blockDim.x) {
    const int r = (int)(it % 128);
    const int k8 = (int)((it / 128) % (d.KP / 8));
    const int64_t t = it / ((int64_t)(d.KP / 8) * 128);
    const int64_t s = t * 128 + r;
    uint16_t v[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int i = 8 * k8 + q;
      v[q] = 0;
      if (s < n && i < d.ns) v[q] = ((bits[s * nw + (i >> 5)] >> (i & 31)) & 1u) ? 0x3F80u : 0xBF80u;
    }
    const int c = (8 * k8) / kKCH, kc = (8 * k8) % kKCH;
    uint8_t* base = reinterpret_cast<uint8_t*>(out) + ((size_t)t * d.nK + c) * (128u * kKCH * 2);
    *reinterpret_cast<uint4*>(base + umma::kmajor_offset(r, kc, 128)) = pk8(v);
  }
}

// W terms: N chunk q, K chunk c, term e -> ((q * nK + c) * 3 + e) * (NR * kKCH * 2) + kmajor(n, k % kKCH, NR)
// row n < NC: Re W of unit q*NC + n; row NC + n (complex): Im W of that unit
template <class T>
__global__ void theta_w_terms_kernel(ThetaDims d, const T* __restrict__ W, uint16_t* __restrict__ out) {
  constexpr bool CPLX = ScalarTraits<T>::is_complex;
  const int64_t items = (int64_t)d.nnc * d.NR * (d.KP / 8);
  const size_t term = (size_t)d.NR * kKCH * 2;
  for (int64_t it = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; it < items; it += (int64_t)gridDim.x * blockDim.x) {
    const int n = (int)(it % d.NR);
    const int k8 = (int)((it / d.NR) % (d.KP / 8));
    const int q = (int)(it / ((int64_t)(d.KP / 8) * d.NR));
    const bool im = CPLX && n >= d.NC;
    const int m = q * d.NC + (im ? n - d.NC : n);
    uint16_t t1[8], t2[8], t3[8];
#pragma unroll
    for (int e = 0; e < 8; ++e) {
      const int i = 8 * k8 + e;
      float x = 0.f;
      if (i < d.ns && m < d.nh) x = im ? wim(W, (int64_t)i * d.nh + m) : wre(W, (int64_t)i * d.nh + m);
      t1[e] = bf(x);
      const float r1 = x - bfv(t1[e]);
      t2[e] = bf(r1);
      t3[e] = bf(r1 - bfv(t2[e]));
    }
    const int c = (8 * k8) / kKCH, kc = (8 * k8) % kKCH;
    uint8_t* base = reinterpret_cast<uint8_t*>(out) + (((size_t)q * d.nK + c) * 3) * term;
    const uint32_t off = umma::kmajor_offset(n, kc, d.NR);
    *reinterpret_cast<uint4*>(base + off) = pk8(t1);
    *reinterpret_cast<uint4*>(base + term + off) = pk8(t2);
    *reinterpret_cast<uint4*>(base + 2 * term + off) = pk8(t3);
  }
}

template <class T>
__global__ void __launch_bounds__(kThr) theta_tc_kernel(ThetaDims d, int64_t n, const uint16_t* __restrict__ sig_rows,
                                                        const uint16_t* __restrict__ wterms, const T* __restrict__ b,
                                                        T* __restrict__ theta_out, T* __restrict__ tanh_out,
                                                        T* __restrict__ lsum_part, int* __restrict__ status) {
  extern __shared__ __align__(128) uint8_t smem[];
  constexpr bool CPLX = ScalarTraits<T>::is_complex;
  const int NR = d.NR, NC = d.NC, nK = d.nK, S = d.stages, nh = d.nh;
  const uint32_t a_bytes = 128u * kKCH * 2u, b_term = (uint32_t)NR * kKCH * 2u;
  const uint32_t stage_bytes = a_bytes + 3u * b_term;
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + S * stage_bytes);
  uint64_t* empty = full + 4;
  uint64_t* done = empty + 4;
  uint32_t* tslot = reinterpret_cast<uint32_t*>(done + 1);
  __shared__ T s_part[kCG][128];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int tile = blockIdx.x, q = blockIdx.y;
  if (tid == 0) {
    for (int k = 0; k < S; ++k) { umma::mbar_init(&full[k], 1); umma::mbar_init(&empty[k], 1); }
    umma::mbar_init(done, 1);
    umma::fence_mbar_init();
  }
  if (warp == 0) {
    umma::tmem_alloc(tslot, d.tmem_cols);
    umma::tmem_relinquish();
  }
  umma::tc_fence_before();
  __syncthreads();
  umma::tc_fence_after();
  const uint32_t tbase = *tslot;
  if (warp == 0 && lane == 0) {
    const uint8_t* ga = reinterpret_cast<const uint8_t*>(sig_rows) + (size_t)tile * nK * a_bytes;
    const uint8_t* gb = reinterpret_cast<const uint8_t*>(wterms) + (size_t)q * nK * 3 * b_term;
    for (int c = 0; c < nK; ++c) {
      const int st = c % S;
      if (c >= S && !umma::mbar_wait(&empty[st], ((c / S) - 1) & 1, kWait)) {
        atomicCAS(status, 0, QES_ERR_TIMEOUT);
        break;
      }
      uint8_t* sp = smem + st * stage_bytes;
      umma::mbar_arrive_expect_tx(&full[st], stage_bytes);
      umma::bulk_g2s(sp, ga + (size_t)c * a_bytes, a_bytes, &full[st]);
      umma::bulk_g2s(sp + a_bytes, gb + (size_t)c * 3 * b_term, 3 * b_term, &full[st]);
    }
  } else if (warp == 1 && lane == 0) {
    const int n_parts = NR > 256 ? 2 : 1;
    const uint32_t np0 = NR > 256 ? 256u : (uint32_t)NR;
    for (int c = 0; c < nK; ++c) {
      const int st = c % S;
      if (!umma::mbar_wait(&full[st], (c / S) & 1, kWait)) {
        atomicCAS(status, 0, QES_ERR_TIMEOUT);
        break;
      }
      umma::tc_fence_after();
      const uint32_t sa = umma::smem_u32(smem + st * stage_bytes);
      const uint32_t sb = sa + a_bytes;
      for (int kk = 0; kk < kKCH / 16; ++kk) {
        const uint64_t da = umma::smem_desc(sa + 2u * kk * 128u * 16u, 128u * 16u, 128u);
        for (int pt = 0; pt < n_parts; ++pt) {
          const uint32_t n0 = pt ? np0 : 0u, nn = pt ? (uint32_t)NR - np0 : np0;
          const uint32_t idesc = umma::idesc_bf16_f32(128, nn);
          for (int e = 0; e < 3; ++e) {
            const uint64_t db = umma::smem_desc(sb + (uint32_t)e * b_term + 2u * kk * NR * 16u + (n0 / 8u) * 128u,
                                                NR * 16u, 128u);
            umma::mma_bf16(tbase + n0, da, db, idesc, (c > 0 || kk > 0 || e > 0) ? 1u : 0u);
          }
        }
      }
      umma::mma_commit(&empty[st]);
    }
    umma::mma_commit(done);
  }
  __syncthreads();
  const bool ok = umma::mbar_wait(done, 0, kWait);
  if (!ok) atomicCAS(status, 0, QES_ERR_TIMEOUT);
  umma::tc_fence_after();
  // epilogue: warp w reads lane quarter w % 4 (samples), column group w / 4 (units)
  const int quarter = warp & 3, cg = warp >> 2;
  const int row = 32 * quarter + lane;
  const int64_t s = (int64_t)tile * 128 + row;
  const bool sval = s < n;
  const uint32_t lane_addr = tbase + ((uint32_t)(32 * quarter) << 16);
  T lsum = ScalarTraits<T>::zero();
  for (int c = cg; ok && c < NC / 16; c += kCG) {
    float re[16], im[16];
    umma::tmem_ld16(lane_addr + 16 * c, re);
    if constexpr (CPLX) umma::tmem_ld16(lane_addr + NC + 16 * c, im);
#pragma unroll
    for (int e = 0; e < 16; ++e) {
      const int m = q * NC + 16 * c + e;
      if (sval && m < nh) {
        T th;
        if constexpr (CPLX) th = make_float2(re[e] + b[m].x, im[e] + b[m].y);
        else th = re[e] + b[m];
        if (theta_out) theta_out[s * nh + m] = th;
        if (tanh_out) tanh_out[s * nh + m] = tanhx(th);
        lsum = addx(lsum, log_cosh(th));
      }
    }
  }
  s_part[cg][row] = lsum;
  umma::tc_fence_before();
  __syncthreads();
  if (cg == 0 && sval && lsum_part) {
    T t = s_part[0][row];
    for (int g = 1; g < kCG; ++g) t = addx(t, s_part[g][row]);
    lsum_part[(int64_t)q * n + s] = t;
  }
  if (warp == 0) umma::tmem_dealloc(tbase, d.tmem_cols);
}

// log psi = sum over N chunks of the log cosh partials + sigma . a
template <class T>
__global__ void theta_logpsi_kernel(int ns, int nnc, int64_t n, const uint32_t* __restrict__ bits,
                                    const T* __restrict__ a, const T* __restrict__ lsum_part, T* __restrict__ logpsi) {
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const uint32_t* w = bits + s * n_words(ns);
  T v = ScalarTraits<T>::zero();
  for (int q = 0; q < nnc; ++q) v = addx(v, lsum_part[(int64_t)q * n + s]);
  for (int i = 0; i < ns; ++i) v = addx(v, scal(sigma_of(w, i), a[i]));
  logpsi[s] = v;
}

static size_t al256t(size_t x) { return (x + 255) & ~(size_t)255; }

static size_t theta_ws(const ThetaDims& d, int64_t n, size_t tsz, size_t* o_w, size_t* o_l, size_t* o_s) {
  const size_t sig = (size_t)d.n_tiles * 128 * d.KP * 2;
  const size_t wt = (size_t)d.nnc * d.nK * 3 * d.NR * kKCH * 2;
  const size_t ls = (size_t)d.nnc * n * tsz;
  *o_w = al256t(sig);
  *o_l = *o_w + al256t(wt);
  *o_s = *o_l + al256t(ls);
  return *o_s + 256;
}

extern "C" int qes_rbm_forward_tc_workspace_bytes(int dtype, int ns, int nh, int64_t n_samples, size_t* bytes) {
  QES_ARG_CHECK(bytes && ns > 0 && nh > 0 && n_samples > 0, "qes_rbm_forward_tc_workspace_bytes: bad args");
  QES_ARG_CHECK(dtype == QES_DTYPE_F32 || dtype == QES_DTYPE_C64, "qes_rbm_forward_tc_workspace_bytes: bad dtype");
  ThetaDims d;
  if (!theta_plan(dtype == QES_DTYPE_C64, ns, nh, n_samples, &d)) {
    qes_set_last_message("qes_rbm_forward_tc: shapes outside the tensor-core forward's limits");
    return QES_ERR_SIZE;
  }
  size_t a, b, c;
  *bytes = theta_ws(d, n_samples, dtype == QES_DTYPE_C64 ? 8 : 4, &a, &b, &c);
  return QES_OK;
}

template <class T>
static int forward_tc_t(const ThetaDims& d, int64_t n, const uint32_t* bits, const T* a, const T* b, const T* W,
                        T* theta_out, T* tanh_out, T* logpsi_out, char* ws, cudaStream_t st) {
  size_t ow, ol, os;
  theta_ws(d, n, sizeof(T), &ow, &ol, &os);
  uint16_t* sig = reinterpret_cast<uint16_t*>(ws);
  uint16_t* wt = reinterpret_cast<uint16_t*>(ws + ow);
  T* lsum = reinterpret_cast<T*>(ws + ol);
  int* status = reinterpret_cast<int*>(ws + os);
  QES_CUDA_CHECK(cudaMemsetAsync(status, 0, sizeof(int), st));
  QES_CUDA_CHECK(cudaFuncSetAttribute(theta_tc_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, d.smem));
  theta_sig_rows_kernel<<<1184, 256, 0, st>>>(d, n, bits, sig);
  theta_w_terms_kernel<T><<<296, 256, 0, st>>>(d, W, wt);
  theta_tc_kernel<T><<<dim3(d.n_tiles, d.nnc), kThr, d.smem, st>>>(d, n, sig, wt, b, theta_out, tanh_out,
                                                                    logpsi_out ? lsum : nullptr, status);
  QES_LAUNCH_CHECK_N(3);
  if (logpsi_out) {
    theta_logpsi_kernel<T><<<(unsigned)((n + 255) / 256), 256, 0, st>>>(d.ns, d.nnc, n, bits, a, lsum, logpsi_out);
    QES_LAUNCH_CHECK();
  }
  int h = 0;
  QES_CUDA_CHECK(cudaMemcpyAsync(&h, status, sizeof(int), cudaMemcpyDeviceToHost, st));
  QES_CUDA_CHECK(cudaStreamSynchronize(st));
  if (h) {
    qes_set_last_message("qes_rbm_forward_tc: a bounded device wait gave up");
    return QES_ERR_TIMEOUT;
  }
  return QES_OK;
}

extern "C" int qes_rbm_forward_tc(int dtype, int ns, int nh, int64_t n_samples, const uint32_t* bits, const void* a,
                                  const void* b, const void* W, void* theta_out, void* tanh_out, void* logpsi_out,
                                  void* workspace, size_t workspace_bytes, void* stream) {
  QES_ARG_CHECK(ns > 0 && nh > 0 && n_samples >= 0, "qes_rbm_forward_tc: bad sizes");
  QES_ARG_CHECK(dtype == QES_DTYPE_F32 || dtype == QES_DTYPE_C64, "qes_rbm_forward_tc: bad dtype");
  if (n_samples == 0) return QES_OK;
  QES_ARG_CHECK(bits && a && b && W && workspace, "qes_rbm_forward_tc: null pointer");
  ThetaDims d;
  if (!theta_plan(dtype == QES_DTYPE_C64, ns, nh, n_samples, &d)) {
    qes_set_last_message("qes_rbm_forward_tc: shapes outside the tensor-core forward's limits");
    return QES_ERR_SIZE;
  }
  size_t x, y, z;
  if (workspace_bytes < theta_ws(d, n_samples, dtype == QES_DTYPE_C64 ? 8 : 4, &x, &y, &z)) {
    qes_set_last_message("qes_rbm_forward_tc: workspace too small");
    return QES_ERR_WORKSPACE;
  }
  cudaStream_t st = (cudaStream_t)stream;
  if (dtype == QES_DTYPE_F32)
    return forward_tc_t<float>(d, n_samples, bits, (const float*)a, (const float*)b, (const float*)W,
                               (float*)theta_out, (float*)tanh_out, (float*)logpsi_out, (char*)workspace, st);
  return forward_tc_t<float2>(d, n_samples, bits, (const float2*)a, (const float2*)b, (const float2*)W,
                              (float2*)theta_out, (float2*)tanh_out, (float2*)logpsi_out, (char*)workspace, st);
}
