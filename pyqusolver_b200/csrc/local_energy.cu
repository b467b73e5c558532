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

template <class T>
__global__ void __launch_bounds__(32 * ELOC_ROWS) eloc_moves_kernel(
    int ns, int nh, int64_t n_samples, const uint32_t* __restrict__ bits, const T* __restrict__ tanh_theta,
    int K, const int32_t* __restrict__ mi, const int32_t* __restrict__ mj, const int32_t* __restrict__ mkind,
    const float4* __restrict__ mcoef, const T* __restrict__ Ct, const T* __restrict__ St,
    const T* __restrict__ A, float2* __restrict__ partial /* [gridDim.x][n_samples] */) {
  const int nw = n_words(ns);
  const int k = blockIdx.x * 32 + threadIdx.x;
  const int64_t s_base = (int64_t)blockIdx.y * ELOC_SB + (int64_t)threadIdx.y * ELOC_SPT;
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
    for (int m0 = 0; m0 < nh; m0 += ELOC_RENORM) {
      const int m1 = min(nh, m0 + ELOC_RENORM);
      for (int m = m0; m < m1; ++m) {
        const T c = Ct[(int64_t)m * K + k];
        const T s = St[(int64_t)m * K + k];
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
      if (s < n_samples) partial[(int64_t)blockIdx.x * n_samples + s] = v;
    }
  }
}

__global__ void eloc_reduce_kernel(int ns, int64_t n_samples, const uint32_t* __restrict__ bits, int nkb,
                                   const float2* __restrict__ partial, int n_zf, const int32_t* __restrict__ zf_site,
                                   const float* __restrict__ zf_h, int n_zz, const int32_t* __restrict__ zz_i,
                                   const int32_t* __restrict__ zz_j, const float* __restrict__ zz_J,
                                   float2* __restrict__ eloc) {
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n_samples) return;
  const int nw = n_words(ns);
  const uint32_t* w = bits + s * nw;
  float d = 0.f;
  for (int t = 0; t < n_zf; ++t) d += zf_h[t] * sigma_of(w, zf_site[t]);
  for (int t = 0; t < n_zz; ++t) d += zz_J[t] * ((bit_of(w, zz_i[t]) == bit_of(w, zz_j[t])) ? 1.f : -1.f);
  float2 e = make_float2(d, 0.f);
  for (int b = 0; b < nkb; ++b) e = e + partial[(int64_t)b * n_samples + s];
  eloc[s] = e;
}

static int eloc_kblocks(int K) { return (K + 31) / 32; }

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
