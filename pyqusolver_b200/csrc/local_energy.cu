// Fused local-energy kernel and float64 energy statistics.
//
// E_loc(s) = diag(s) + sum_k active_k(s) conj(c_k(s)) exp(-2 sigma_i A_k)
//                        prod_m (C_km - sigma_i tanh(theta_sm) S_km)
//
// The reference evaluates the full network on every connected state
// (O(K*N*M) per sample); here each psi ratio is a product over hidden units
// of one complex FMA against per-move tables that depend only on W, so the
// work is O(K*M) per sample with no transcendental in the inner loop.
//
// Mapping: block = 32 moves (threadIdx.x, one warp row) x ELOC_ROWS sample
// groups (threadIdx.y) of ELOC_SPT samples each.  Tables are stored m-major
// (Ct[m][k]) so a warp reads 32 consecutive moves of one hidden unit per
// load; tanh(theta) rows are warp-broadcast.  Each block writes one partial
// sum per sample (deterministic), reduced by eloc_reduce_kernel together with
// the diagonal part.
#include "common.cuh"

#define QES_ARG_CHECK(cond, msg) do { if (!(cond)) { qes_set_last_message(msg); return QES_ERR_ARG; } } while (0)

constexpr int ELOC_SPT = 4;     // samples per thread
constexpr int ELOC_ROWS = 8;    // sample groups per block
constexpr int ELOC_SB = ELOC_SPT * ELOC_ROWS;   // samples per block
constexpr int ELOC_RENORM = 16; // hidden units between renormalisations

// Move block kb (32 moves) x sample block sb (ELOC_SB samples) of one problem.
template <class T>
QES_D void eloc_moves_block(int kb, int64_t sb, int ns, int nh, int64_t n_samples, const uint32_t* __restrict__ bits,
                            const T* __restrict__ tanh_theta, int K, const int32_t* __restrict__ mi,
                            const int32_t* __restrict__ mj, const int32_t* __restrict__ mkind,
                            const float4* __restrict__ mcoef, const T* __restrict__ Ct, const T* __restrict__ St,
                            const T* __restrict__ A, float2* __restrict__ partial /* [kblocks][n_samples] */) {
  const int nw = n_words(ns);
  const int k = kb * 32 + threadIdx.x;
  const int64_t s_base = sb * ELOC_SB + (int64_t)threadIdx.y * ELOC_SPT;
  const bool kval = k < K;

  int kind = 0, i = 0, j = 0;
  float4 cf = make_float4(0.f, 0.f, 0.f, 0.f);
  T Ak = ScalarTraits<T>::zero();
  if (kval) {
    kind = mkind[k]; i = mi[k]; j = mj[k]; cf = mcoef[k]; Ak = A[k];
  }

  float g[ELOC_SPT];        // -sigma_i per sample
  bool act[ELOC_SPT];
  const T* trow[ELOC_SPT];
#pragma unroll
  for (int q = 0; q < ELOC_SPT; ++q) {
    const int64_t s = s_base + q;
    const bool sval = s < n_samples;
    const int64_t sc = sval ? s : 0;
    const uint32_t* w = bits + sc * nw;
    const uint32_t bi = kval ? bit_of(w, i) : 0u;
    bool a = kval && sval;
    if (kind == QES_MOVE_PAIR_ANTI) a = a && (bit_of(w, j) != bi);
    else if (kind == QES_MOVE_PAIR_PAR) a = a && (bit_of(w, j) == bi);
    act[q] = a;
    g[q] = bi ? -1.f : 1.f;
    trow[q] = tanh_theta + sc * nh;
  }

  T acc[ELOC_SPT];
  int ex[ELOC_SPT];
#pragma unroll
  for (int q = 0; q < ELOC_SPT; ++q) { acc[q] = ScalarTraits<T>::one(); ex[q] = 0; }

  if (kval) {
    // whole blocks of ELOC_RENORM units unrolled, then the tail; the same factor order and the same
    // renormalisation points as one loop over m
    const T* cp = Ct + k;
    const T* sp = St + k;
    int m0 = 0;
    for (; m0 + ELOC_RENORM <= nh; m0 += ELOC_RENORM) {
#pragma unroll
      for (int u = 0; u < ELOC_RENORM; ++u) {
        const int m = m0 + u;
        const T c = cp[(int64_t)m * K];
        const T s = sp[(int64_t)m * K];
#pragma unroll
        for (int q = 0; q < ELOC_SPT; ++q) acc[q] = mulx(acc[q], ratio_factor(c, g[q], trow[q][m], s));
      }
#pragma unroll
      for (int q = 0; q < ELOC_SPT; ++q) renorm(acc[q], ex[q]);
    }
    if (m0 < nh) {
      for (int m = m0; m < nh; ++m) {
        const T c = cp[(int64_t)m * K];
        const T s = sp[(int64_t)m * K];
#pragma unroll
        for (int q = 0; q < ELOC_SPT; ++q) acc[q] = mulx(acc[q], ratio_factor(c, g[q], trow[q][m], s));
      }
#pragma unroll
      for (int q = 0; q < ELOC_SPT; ++q) renorm(acc[q], ex[q]);
    }
  }

  // contribution = coef * exp(g*2*A + ex*ln2) * acc   (g = -sigma_i)
#pragma unroll
  for (int q = 0; q < ELOC_SPT; ++q) {
    float2 v = make_float2(0.f, 0.f);
    if (act[q]) {
      const float sig = -g[q];
      const float2 coef = make_float2(cf.x + sig * cf.z, cf.y + sig * cf.w);
      // exp(-2 sigma_i A_k) with the power-of-two exponent folded into the modulus
      const float2 z = to_c(scal(2.f * g[q], Ak));
      const float2 e = to_c(expx(make_float2(z.x + 0.69314718055994531f * (float)ex[q], z.y)));
      v = coef * (e * to_c(acc[q]));
    }
    v = warp_sum(v);
    if (threadIdx.x == 0) {
      const int64_t s = s_base + q;
      if (s < n_samples) partial[(int64_t)kb * n_samples + s] = v;
    }
  }
}

template <class T>
__global__ void __launch_bounds__(32 * ELOC_ROWS) eloc_moves_kernel(
    int ns, int nh, int64_t n_samples, const uint32_t* __restrict__ bits, const T* __restrict__ tanh_theta,
    int K, const int32_t* __restrict__ mi, const int32_t* __restrict__ mj, const int32_t* __restrict__ mkind,
    const float4* __restrict__ mcoef, const T* __restrict__ Ct, const T* __restrict__ St,
    const T* __restrict__ A, float2* __restrict__ partial /* [gridDim.x][n_samples] */) {
  eloc_moves_block<T>(blockIdx.x, blockIdx.y, ns, nh, n_samples, bits, tanh_theta, K, mi, mj, mkind, mcoef, Ct, St, A,
                      partial);
}

// diagonal part + move partials of sample s
QES_D void eloc_reduce_sample(int64_t s, int ns, int64_t n_samples, const uint32_t* __restrict__ bits, int nkb,
                              const float2* __restrict__ partial, int n_zf, const int32_t* __restrict__ zf_site,
                              const float* __restrict__ zf_h, int n_zz, const int32_t* __restrict__ zz_i,
                              const int32_t* __restrict__ zz_j, const float* __restrict__ zz_J,
                              float2* __restrict__ eloc) {
  const int nw = n_words(ns);
  const uint32_t* w = bits + s * nw;
  float d = 0.f;
  for (int t = 0; t < n_zf; ++t) d += zf_h[t] * sigma_of(w, zf_site[t]);
  for (int t = 0; t < n_zz; ++t) d += zz_J[t] * ((bit_of(w, zz_i[t]) == bit_of(w, zz_j[t])) ? 1.f : -1.f);
  float2 e = make_float2(d, 0.f);
  for (int b = 0; b < nkb; ++b) e = e + partial[(int64_t)b * n_samples + s];
  eloc[s] = e;
}

__global__ void eloc_reduce_kernel(int ns, int64_t n_samples, const uint32_t* __restrict__ bits, int nkb,
                                   const float2* __restrict__ partial, int n_zf, const int32_t* __restrict__ zf_site,
                                   const float* __restrict__ zf_h, int n_zz, const int32_t* __restrict__ zz_i,
                                   const int32_t* __restrict__ zz_j, const float* __restrict__ zz_J,
                                   float2* __restrict__ eloc) {
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n_samples) return;
  eloc_reduce_sample(s, ns, n_samples, bits, nkb, partial, n_zf, zf_site, zf_h, n_zz, zz_i, zz_j, zz_J, eloc);
}

QES_HD int eloc_kblocks(int K) { return (K + 31) / 32; }

extern "C" int qes_local_energy_workspace_bytes(int dtype, int ns, int nh, int64_t n_samples, int n_moves,
                                                size_t* bytes) {
  QES_ARG_CHECK(bytes != nullptr && n_samples >= 0 && n_moves >= 0, "qes_local_energy_workspace_bytes: bad args");
  (void)dtype; (void)ns; (void)nh;
  *bytes = (size_t)eloc_kblocks(n_moves) * (size_t)n_samples * sizeof(float2);
  return QES_OK;
}

extern "C" int qes_local_energy(int dtype, int ns, int nh, int64_t n_samples, const uint32_t* bits,
                                const void* tanh_theta, const qes_hamiltonian* ham, const void* Ct, const void* St,
                                const void* A, void* workspace, size_t workspace_bytes, void* eloc_out,
                                void* stream) {
  QES_ARG_CHECK(ham != nullptr && ns > 0 && nh > 0 && n_samples >= 0, "qes_local_energy: bad sizes");
  QES_ARG_CHECK(dtype == QES_DTYPE_F32 || dtype == QES_DTYPE_C64, "qes_local_energy: bad dtype");
  if (n_samples == 0) return QES_OK;
  QES_ARG_CHECK(bits && eloc_out, "qes_local_energy: null pointer");
  const int K = ham->n_moves;
  size_t need = 0;
  qes_local_energy_workspace_bytes(dtype, ns, nh, n_samples, K, &need);
  if (workspace_bytes < need || (need > 0 && workspace == nullptr)) {
    qes_set_last_message("qes_local_energy: workspace too small");
    return QES_ERR_WORKSPACE;
  }
  cudaStream_t st = (cudaStream_t)stream;
  const int nkb = eloc_kblocks(K);
  float2* partial = (float2*)workspace;
  if (K > 0) {
    QES_ARG_CHECK(tanh_theta && Ct && St && A && ham->move_i && ham->move_j && ham->move_kind && ham->move_coef,
                  "qes_local_energy: null move pointer");
    const int64_t nsb = (n_samples + ELOC_SB - 1) / ELOC_SB;
    QES_ARG_CHECK(nsb <= 65535, "qes_local_energy: too many samples for one launch");
    dim3 grid(nkb, (unsigned)nsb), block(32, ELOC_ROWS);
    if (dtype == QES_DTYPE_F32)
      eloc_moves_kernel<float><<<grid, block, 0, st>>>(ns, nh, n_samples, bits, (const float*)tanh_theta, K,
                                                       ham->move_i, ham->move_j, ham->move_kind,
                                                       (const float4*)ham->move_coef, (const float*)Ct,
                                                       (const float*)St, (const float*)A, partial);
    else
      eloc_moves_kernel<float2><<<grid, block, 0, st>>>(ns, nh, n_samples, bits, (const float2*)tanh_theta, K,
                                                        ham->move_i, ham->move_j, ham->move_kind,
                                                        (const float4*)ham->move_coef, (const float2*)Ct,
                                                        (const float2*)St, (const float2*)A, partial);
    QES_LAUNCH_CHECK();
  }
  const int bs = 256;
  eloc_reduce_kernel<<<(unsigned)((n_samples + bs - 1) / bs), bs, 0, st>>>(
      ns, n_samples, bits, K > 0 ? nkb : 0, partial, ham->n_zfield, ham->zf_site, ham->zf_h, ham->n_zz, ham->zz_i,
      ham->zz_j, ham->zz_J, (float2*)eloc_out);
  QES_LAUNCH_CHECK();
  return QES_OK;
}

// ----------------------------------------------------------------------------
// float64 statistics of E_loc: mean (complex), variance and std of E_loc,
// Kahan-compensated per thread, then a fixed-order block tree.
// ----------------------------------------------------------------------------
constexpr int STATS_THREADS = 256;
constexpr int STATS_BLOCKS = 148;

__global__ void stats_pass1(int64_t n, const float2* __restrict__ e, const float* __restrict__ w,
                            double* __restrict__ part /* [blocks][4] : sw, swre, swim */) {
  double s0 = 0, s1 = 0, s2 = 0, c0 = 0, c1 = 0, c2 = 0;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
    const double wk = w ? (double)w[k] : 1.0;
    const double y0 = wk - c0, y1 = wk * (double)e[k].x - c1, y2 = wk * (double)e[k].y - c2;
    const double t0 = s0 + y0, t1 = s1 + y1, t2 = s2 + y2;
    c0 = (t0 - s0) - y0; c1 = (t1 - s1) - y1; c2 = (t2 - s2) - y2;
    s0 = t0; s1 = t1; s2 = t2;
  }
  __shared__ double red[3][STATS_THREADS];
  red[0][threadIdx.x] = s0; red[1][threadIdx.x] = s1; red[2][threadIdx.x] = s2;
  __syncthreads();
  for (int o = STATS_THREADS / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o)
      for (int q = 0; q < 3; ++q) red[q][threadIdx.x] += red[q][threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int q = 0; q < 3; ++q) part[blockIdx.x * 4 + q] = red[q][0];
}

__global__ void stats_mean(int nb, int64_t n, const double* __restrict__ part, double* __restrict__ out) {
  if (threadIdx.x != 0) return;
  double s1 = 0, s2 = 0;
  for (int b = 0; b < nb; ++b) { s1 += part[b * 4 + 1]; s2 += part[b * 4 + 2]; }
  out[0] = s1 / (double)n;   // weights are normalised to sum n
  out[1] = s2 / (double)n;
}

__global__ void stats_pass2(int64_t n, const float2* __restrict__ e, const float* __restrict__ w,
                            const double* __restrict__ mean, double* __restrict__ part) {
  const double mr = mean[0], mi = mean[1];
  double s = 0, c = 0;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
    const double wk = w ? (double)w[k] : 1.0;
    const double dr = (double)e[k].x - mr, di = (double)e[k].y - mi;
    const double y = wk * (dr * dr + di * di) - c;
    const double t = s + y;
    c = (t - s) - y;
    s = t;
  }
  __shared__ double red[STATS_THREADS];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int o = STATS_THREADS / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x * 4 + 3] = red[0];
}

__global__ void stats_final(int nb, int64_t n, const double* __restrict__ part, double* __restrict__ out) {
  if (threadIdx.x != 0) return;
  double v = 0;
  for (int b = 0; b < nb; ++b) v += part[b * 4 + 3];
  v /= (double)n;
  out[2] = v;
  out[3] = sqrt(v);
}

extern "C" int qes_loss_stats_workspace_bytes(int64_t n_samples, size_t* bytes) {
  QES_ARG_CHECK(bytes != nullptr && n_samples >= 0, "qes_loss_stats_workspace_bytes: bad args");
  *bytes = (size_t)STATS_BLOCKS * 4 * sizeof(double);
  return QES_OK;
}

extern "C" int qes_loss_stats(int64_t n_samples, const void* eloc, const float* probs, double* out, void* workspace,
                              size_t workspace_bytes, void* stream) {
  QES_ARG_CHECK(n_samples > 0 && eloc && out, "qes_loss_stats: bad args");
  if (workspace_bytes < (size_t)STATS_BLOCKS * 4 * sizeof(double) || !workspace) {
    qes_set_last_message("qes_loss_stats: workspace too small");
    return QES_ERR_WORKSPACE;
  }
  cudaStream_t st = (cudaStream_t)stream;
  double* part = (double*)workspace;
  stats_pass1<<<STATS_BLOCKS, STATS_THREADS, 0, st>>>(n_samples, (const float2*)eloc, probs, part);
  stats_mean<<<1, 32, 0, st>>>(STATS_BLOCKS, n_samples, part, out);
  stats_pass2<<<STATS_BLOCKS, STATS_THREADS, 0, st>>>(n_samples, (const float2*)eloc, probs, out, part);
  stats_final<<<1, 32, 0, st>>>(STATS_BLOCKS, n_samples, part, out);
  QES_LAUNCH_CHECK_N(4);
  return QES_OK;
}

// ----------------------------------------------------------------------------
// Step diagnostics: Gelman-Rubin R-hat over n_groups contiguous blocks of
// Re E_loc and sigma^2 = var(Re E_loc) (uniform weights, ddof 0), float64.
// One warp per block computes its mean and ddof-1 variance (two passes); a
// single CTA then combines the blocks in a fixed order.
// ----------------------------------------------------------------------------
constexpr int RHAT_FINAL_THREADS = 1024;

__global__ void rhat_groups_kernel(int64_t n_groups, int64_t glen, const float2* __restrict__ e,
                                   double2* __restrict__ gstat) {
  const int lane = threadIdx.x & 31;
  const int64_t g = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (g >= n_groups) return;
  const float2* x = e + g * glen;
  double s = 0;
  for (int64_t k = lane; k < glen; k += 32) s += (double)x[k].x;
  const double m = warp_sum(s) / (double)glen;
  double v = 0;
  for (int64_t k = lane; k < glen; k += 32) {
    const double d = (double)x[k].x - m;
    v += d * d;
  }
  v = warp_sum(v);
  if (lane == 0) gstat[g] = make_double2(m, glen > 1 ? v / (double)(glen - 1) : 0.0);
}

__global__ void __launch_bounds__(RHAT_FINAL_THREADS) rhat_final_kernel(int64_t n_groups, int64_t glen, int valid,
                                                                      const double2* __restrict__ gstat,
                                                                      double* __restrict__ out) {
  __shared__ double red[2][RHAT_FINAL_THREADS];
  double sm = 0, sv = 0;
  for (int64_t g = threadIdx.x; g < n_groups; g += blockDim.x) { sm += gstat[g].x; sv += gstat[g].y; }
  red[0][threadIdx.x] = sm; red[1][threadIdx.x] = sv;
  __syncthreads();
  for (int o = RHAT_FINAL_THREADS / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) { red[0][threadIdx.x] += red[0][threadIdx.x + o]; red[1][threadIdx.x] += red[1][threadIdx.x + o]; }
    __syncthreads();
  }
  const double mm = red[0][0] / (double)n_groups;   // grand mean (equal block lengths)
  const double W = red[1][0] / (double)n_groups;    // mean within-block variance
  __syncthreads();
  double sb = 0;
  for (int64_t g = threadIdx.x; g < n_groups; g += blockDim.x) {
    const double d = gstat[g].x - mm;
    sb += d * d;
  }
  red[0][threadIdx.x] = sb;
  __syncthreads();
  for (int o = RHAT_FINAL_THREADS / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[0][threadIdx.x] += red[0][threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const double L = (double)glen, G = (double)n_groups, ssb = red[0][0];
    // total variance of the n = G*L values, ddof 0: within + between blocks
    out[1] = ((L - 1.0) * W * G + L * ssb) / (G * L);
    if (valid) {
      const double B = L * ssb / (G - 1.0);
      const double var_hat = ((L - 1.0) / L) * W + B / L;
      out[0] = sqrt(var_hat / fmax(W, 1e-12));
    } else {
      out[0] = nan("");
    }
  }
}

extern "C" int qes_loss_rhat_workspace_bytes(int64_t n_samples, int n_chains, size_t* bytes) {
  QES_ARG_CHECK(bytes != nullptr && n_samples >= 0, "qes_loss_rhat_workspace_bytes: bad args");
  *bytes = (size_t)std::max<int64_t>(1, std::max<int64_t>(n_chains, 1)) * sizeof(double2);
  return QES_OK;
}

extern "C" int qes_loss_rhat(int64_t n_samples, int n_chains, const void* eloc, double* out, void* workspace,
                             size_t workspace_bytes, void* stream) {
  QES_ARG_CHECK(n_samples > 0 && eloc && out && workspace, "qes_loss_rhat: bad args");
  const int64_t nch = std::max(n_chains, 1);
  const bool valid = nch > 1 && n_samples > nch && n_samples % nch == 0 && n_samples / nch > 1;
  const int64_t G = valid ? nch : 1, L = n_samples / G;
  if (workspace_bytes < (size_t)G * sizeof(double2)) {
    qes_set_last_message("qes_loss_rhat: workspace too small");
    return QES_ERR_WORKSPACE;
  }
  cudaStream_t st = (cudaStream_t)stream;
  double2* gstat = (double2*)workspace;
  const int warps = 8;
  rhat_groups_kernel<<<(unsigned)((G + warps - 1) / warps), 32 * warps, 0, st>>>(G, L, (const float2*)eloc, gstat);
  rhat_final_kernel<<<1, RHAT_FINAL_THREADS, 0, st>>>(G, L, valid ? 1 : 0, gstat, out);
  QES_LAUNCH_CHECK_N(2);
  return QES_OK;
}

// ----------------------------------------------------------------------------
// Allocation-free local energy.
//
// Some callers cannot allocate device memory at all: hosts that hand this
// library a fixed device budget at start-up and forbid cudaMalloc afterwards,
// latency-critical loops where cudaMalloc's implicit device synchronisation is
// not acceptable, and foreign-language bindings (cgo, JNI, plain C) that have
// no allocator of their own to hand out scratch buffers.  For them this entry
// point keeps the local energy's only scratch -- one float2 partial sum per
// (32-move block, sample) -- in a fixed array compiled into the library.
//
// The array lives in every GPU that loads the library until the process
// exits.  The host never dereferences the symbol itself: the array's device
// address is looked up with cudaGetSymbolAddress on the first call made on
// each device (with that device current) and cached, so that first call per
// device should come before any stream capture.  All calls share the one
// array: each call overwrites the part it reads before reading it, so no
// clearing is needed, but calls that overlap on the GPU (several streams or
// host threads at once) race on it and must be serialised by the caller.
// ----------------------------------------------------------------------------
#include <mutex>

static __device__ __align__(256) float2 g_eloc_noalloc_scratch[QES_NOALLOC_ELOC_SCRATCH_BYTES / sizeof(float2)];

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
void* g_noalloc_ptr[kMaxDevices] = {};
}  // namespace

static int eloc_noalloc_scratch(void** out) {
  int dev = -1;
  QES_CUDA_CHECK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) {
    qes_set_last_message("qes_local_energy_noalloc: device ordinal beyond the supported 64");
    return QES_ERR_SIZE;
  }
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (g_noalloc_ptr[dev] == nullptr) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_eloc_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr) {
      qes_set_last_error(e, "qes_local_energy_noalloc: cudaGetSymbolAddress of the static scratch");
      return QES_ERR_CUDA;
    }
    g_noalloc_ptr[dev] = p;
  }
  *out = g_noalloc_ptr[dev];
  return QES_OK;
}

extern "C" int qes_local_energy_noalloc(int dtype, int ns, int nh, int64_t n_samples, const uint32_t* bits,
                                        const void* tanh_theta, const qes_hamiltonian* ham, const void* Ct,
                                        const void* St, const void* A, void* eloc_out, void* stream) {
  QES_ARG_CHECK(ham != nullptr && ns > 0 && nh > 0 && n_samples >= 0, "qes_local_energy_noalloc: bad sizes");
  size_t need = 0;
  const int rc0 = qes_local_energy_workspace_bytes(dtype, ns, nh, n_samples, ham->n_moves, &need);
  if (rc0 != QES_OK) return rc0;
  if (need > (size_t)QES_NOALLOC_ELOC_SCRATCH_BYTES) {
    qes_set_last_message("qes_local_energy_noalloc: ceil(n_moves/32) * n_samples * 8 bytes exceeds the "
                         "8 MiB static scratch; use qes_local_energy with a caller workspace");
    return QES_ERR_SIZE;
  }
  void* scratch = nullptr;
  const int rc = eloc_noalloc_scratch(&scratch);
  if (rc != QES_OK) return rc;
  return qes_local_energy(dtype, ns, nh, n_samples, bits, tanh_theta, ham, Ct, St, A, scratch,
                          (size_t)QES_NOALLOC_ELOC_SCRATCH_BYTES, eloc_out, stream);
}

// ----------------------------------------------------------------------------
// Batched problems
// ----------------------------------------------------------------------------
// move items (b, move block, sample block)
template <class T>
__global__ void __launch_bounds__(32 * ELOC_ROWS) batch_eloc_moves_kernel(
    const qes_batch_instance* __restrict__ inst, const int4* __restrict__ items, const uint32_t* __restrict__ bits,
    const T* __restrict__ tanh_theta, const int32_t* __restrict__ mi, const int32_t* __restrict__ mj,
    const int32_t* __restrict__ mkind, const float4* __restrict__ mcoef, const T* __restrict__ Ct,
    const T* __restrict__ St, const T* __restrict__ A, float2* __restrict__ partial) {
  const int4 it = items[blockIdx.x];
  const qes_batch_instance I = inst[it.x];
  const int64_t rows = (int64_t)I.n_chains * I.num_samples;
  eloc_moves_block<T>(it.y, it.z, I.ns, I.nh, rows, bits + I.sample_word_off, tanh_theta + I.tanh_off, I.n_moves,
                      mi + I.move_off, mj + I.move_off, mkind + I.move_off, mcoef + I.move_off,
                      Ct + I.move_table_off, St + I.move_table_off, A + I.move_off, partial + I.eloc_part_off);
}

// reduce items (b, sample block of 256)
__global__ void batch_eloc_reduce_kernel(const qes_batch_instance* __restrict__ inst, const int4* __restrict__ items,
                                         const uint32_t* __restrict__ bits, const float2* __restrict__ partial,
                                         const int32_t* __restrict__ zf_site, const float* __restrict__ zf_h,
                                         const int32_t* __restrict__ zz_i, const int32_t* __restrict__ zz_j,
                                         const float* __restrict__ zz_J, float2* __restrict__ eloc) {
  const int4 it = items[blockIdx.x];
  const qes_batch_instance I = inst[it.x];
  const int64_t rows = (int64_t)I.n_chains * I.num_samples;
  const int64_t s = (int64_t)it.y * blockDim.x + threadIdx.x;
  if (s >= rows) return;
  eloc_reduce_sample(s, I.ns, rows, bits + I.sample_word_off, I.n_moves > 0 ? eloc_kblocks(I.n_moves) : 0,
                     partial + I.eloc_part_off, I.n_zfield, zf_site + I.zf_off, zf_h + I.zf_off, I.n_zz,
                     zz_i + I.zz_off, zz_j + I.zz_off, zz_J + I.zz_off, eloc + I.sample_off);
}

extern "C" int qes_batch_local_energy(int dtype, int n_inst, const qes_batch_instance* inst, int n_move_items,
                                      const int32_t* move_items, int n_red_items, const int32_t* red_items,
                                      const uint32_t* sample_bits, const void* tanh_theta, const int32_t* move_i,
                                      const int32_t* move_j, const int32_t* move_kind, const float* move_coef,
                                      const void* Ct, const void* St, const void* A, const int32_t* zf_site,
                                      const float* zf_h, const int32_t* zz_i, const int32_t* zz_j,
                                      const float* zz_J, void* partial, void* eloc_out, void* stream) {
  QES_ARG_CHECK(dtype == QES_DTYPE_F32 || dtype == QES_DTYPE_C64, "qes_batch_local_energy: bad dtype");
  QES_ARG_CHECK(n_inst >= 0 && n_move_items >= 0 && n_red_items >= 0, "qes_batch_local_energy: bad sizes");
  if (n_red_items == 0) return QES_OK;
  QES_ARG_CHECK(inst && red_items && sample_bits && eloc_out, "qes_batch_local_energy: null pointer");
  cudaStream_t st = (cudaStream_t)stream;
  if (n_move_items > 0) {
    QES_ARG_CHECK(move_items && tanh_theta && move_i && move_j && move_kind && move_coef && Ct && St && A && partial,
                  "qes_batch_local_energy: null move pointer");
    dim3 block(32, ELOC_ROWS);
    if (dtype == QES_DTYPE_F32)
      batch_eloc_moves_kernel<float><<<n_move_items, block, 0, st>>>(
          inst, (const int4*)move_items, sample_bits, (const float*)tanh_theta, move_i, move_j, move_kind,
          (const float4*)move_coef, (const float*)Ct, (const float*)St, (const float*)A, (float2*)partial);
    else
      batch_eloc_moves_kernel<float2><<<n_move_items, block, 0, st>>>(
          inst, (const int4*)move_items, sample_bits, (const float2*)tanh_theta, move_i, move_j, move_kind,
          (const float4*)move_coef, (const float2*)Ct, (const float2*)St, (const float2*)A, (float2*)partial);
    QES_LAUNCH_CHECK();
  }
  batch_eloc_reduce_kernel<<<n_red_items, 256, 0, st>>>(inst, (const int4*)red_items, sample_bits,
                                                        (const float2*)partial, zf_site, zf_h, zz_i, zz_j, zz_J,
                                                        (float2*)eloc_out);
  QES_LAUNCH_CHECK();
  return QES_OK;
}

// one block per problem: float64 mean (complex), variance, std of its E_loc rows (uniform weights)
constexpr int BSTAT_THREADS = 256;
__global__ void __launch_bounds__(BSTAT_THREADS) batch_stats_kernel(const qes_batch_instance* __restrict__ inst,
                                                                   const float2* __restrict__ eloc,
                                                                   double* __restrict__ out) {
  const qes_batch_instance I = inst[blockIdx.x];
  const int64_t rows = (int64_t)I.n_chains * I.num_samples;
  const float2* e = eloc + I.sample_off;
  __shared__ double red[2][BSTAT_THREADS];
  double sr = 0, si = 0;
  for (int64_t k = threadIdx.x; k < rows; k += blockDim.x) { sr += e[k].x; si += e[k].y; }
  red[0][threadIdx.x] = sr; red[1][threadIdx.x] = si;
  __syncthreads();
  for (int o = BSTAT_THREADS / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) { red[0][threadIdx.x] += red[0][threadIdx.x + o]; red[1][threadIdx.x] += red[1][threadIdx.x + o]; }
    __syncthreads();
  }
  const double n = (double)(rows > 0 ? rows : 1);
  const double mr = red[0][0] / n, mi = red[1][0] / n;
  __syncthreads();
  double v = 0;
  for (int64_t k = threadIdx.x; k < rows; k += blockDim.x) {
    const double dr = e[k].x - mr, di = e[k].y - mi;
    v += dr * dr + di * di;
  }
  red[0][threadIdx.x] = v;
  __syncthreads();
  for (int o = BSTAT_THREADS / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[0][threadIdx.x] += red[0][threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const double var = red[0][0] / n;
    out[4 * blockIdx.x + 0] = mr;
    out[4 * blockIdx.x + 1] = mi;
    out[4 * blockIdx.x + 2] = var;
    out[4 * blockIdx.x + 3] = sqrt(var);
  }
}

extern "C" int qes_batch_loss_stats(int n_inst, const qes_batch_instance* inst, const void* eloc, double* out,
                                    void* stream) {
  QES_ARG_CHECK(n_inst >= 0, "qes_batch_loss_stats: bad sizes");
  if (n_inst == 0) return QES_OK;
  QES_ARG_CHECK(inst && eloc && out, "qes_batch_loss_stats: null pointer");
  batch_stats_kernel<<<n_inst, BSTAT_THREADS, 0, (cudaStream_t)stream>>>(inst, (const float2*)eloc, out);
  QES_LAUNCH_CHECK();
  return QES_OK;
}
