// RBM kernels: initial chains, ratio tables, forward (theta / tanh / log psi),
// log-derivatives and the float64 parameter update.
#include "common.cuh"

#include <stdio.h>
#include <string.h>
#include <algorithm>
#include <atomic>

static thread_local char g_last_error[512] = "";

void qes_set_last_error(cudaError_t e, const char* what) {
  snprintf(g_last_error, sizeof(g_last_error), "%s: %s", what, cudaGetErrorString(e));
}
void qes_set_last_message(const char* msg) { snprintf(g_last_error, sizeof(g_last_error), "%s", msg); }

static std::atomic<long long> g_launches{0};
void qes_count_launches(int n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

static std::atomic<int> g_pdl{1};
bool qes_pdl_on() { return g_pdl.load(std::memory_order_relaxed) != 0; }
extern "C" int qes_set_pdl(int on) {
  g_pdl.store(on ? 1 : 0);
  return QES_OK;
}

extern "C" const char* qes_last_error(void) { return g_last_error; }

// ---------------------------------------------------------------- per-kernel event timing
#include <mutex>
#include <vector>
namespace {
// Event pairs are created on demand in blocks and kept for reuse; between two reads at most
// kProfMaxSlots launches are recorded (later ones are skipped, never blocked on).
constexpr int kProfBlock = 4096;
constexpr int kProfMaxSlots = 1 << 20;
std::mutex g_prof_mu;
std::atomic<int> g_prof_enabled{0};
std::vector<cudaEvent_t> g_prof_ev;   // 2 per slot
std::vector<int> g_prof_cls;
int g_prof_used = 0;
double g_prof_ms[QES_PROF_CLASSES];
long long g_prof_cnt[QES_PROF_CLASSES];

bool prof_grow() {
  const size_t have = g_prof_cls.size();
  if ((int)have >= kProfMaxSlots) return false;
  for (int q = 0; q < kProfBlock; ++q) {
    cudaEvent_t a, b;
    if (cudaEventCreate(&a) != cudaSuccess) return false;
    if (cudaEventCreate(&b) != cudaSuccess) { cudaEventDestroy(a); return false; }
    g_prof_ev.push_back(a);
    g_prof_ev.push_back(b);
    g_prof_cls.push_back(0);
  }
  return true;
}
}  // namespace

bool qes_prof_on() { return g_prof_enabled.load(std::memory_order_relaxed) != 0; }

int qes_prof_begin(int cls, cudaStream_t st) {
  if (!qes_prof_on()) return -1;
  std::lock_guard<std::mutex> lock(g_prof_mu);
  if (g_prof_used >= (int)g_prof_cls.size() && !prof_grow()) return -1;
  const int slot = g_prof_used++;
  g_prof_cls[slot] = cls;
  if (cudaEventRecord(g_prof_ev[2 * slot], st) != cudaSuccess) return -1;
  return slot;
}

void qes_prof_end(int slot, cudaStream_t st) {
  if (slot < 0) return;
  std::lock_guard<std::mutex> lock(g_prof_mu);
  cudaEventRecord(g_prof_ev[2 * slot + 1], st);
}

// folds the recorded pairs into the totals (the caller has synchronised)
static void prof_collect() {
  for (int q = 0; q < g_prof_used; ++q) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, g_prof_ev[2 * q], g_prof_ev[2 * q + 1]) == cudaSuccess) {
      g_prof_ms[g_prof_cls[q]] += ms;
      g_prof_cnt[g_prof_cls[q]] += 1;
    }
  }
  g_prof_used = 0;
}

extern "C" int qes_profile_enable(int enable) {
  std::lock_guard<std::mutex> lock(g_prof_mu);
  if (enable && g_prof_cls.empty() && !prof_grow()) {
    qes_set_last_message("qes_profile_enable: cannot create CUDA events");
    return QES_ERR_CUDA;
  }
  g_prof_enabled.store(enable ? 1 : 0);
  return QES_OK;
}

extern "C" int qes_profile_read(int reset, double* total_ms, long long* counts, int n) {
  std::lock_guard<std::mutex> lock(g_prof_mu);
  QES_CUDA_CHECK(cudaDeviceSynchronize());
  prof_collect();
  for (int k = 0; k < n && k < QES_PROF_CLASSES; ++k) {
    if (total_ms) total_ms[k] = g_prof_ms[k];
    if (counts) counts[k] = g_prof_cnt[k];
  }
  if (reset)
    for (int k = 0; k < QES_PROF_CLASSES; ++k) { g_prof_ms[k] = 0.0; g_prof_cnt[k] = 0; }
  return QES_OK;
}
extern "C" long long qes_launch_count(int reset) {
  return reset ? g_launches.exchange(0) : g_launches.load();
}
extern "C" int qes_version(void) { return 100; }

#define QES_ARG_CHECK(cond, msg) do { if (!(cond)) { qes_set_last_message(msg); return QES_ERR_ARG; } } while (0)

// ----------------------------------------------------------------------------
// initial chains
// ----------------------------------------------------------------------------
__global__ void init_chains_kernel(int kind, int n_up, uint32_t k0, uint32_t k1, int64_t chain_offset,
                                   int n_chains, int ns, uint32_t* __restrict__ out) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n_chains) return;
  const int nw = n_words(ns);
  uint32_t* w = out + (int64_t)c * nw;
  const uint32_t cid = (uint32_t)(chain_offset + c);
  if (kind == QES_INIT_RND) {
    for (int q = 0; q < nw; ++q) {
      Philox4 r = philox4x32_10(cid, (uint32_t)q, 0u, QES_STREAM_INIT_RND, k0, k1);
      uint32_t v = r.x;
      const int rem = ns - 32 * q;
      if (rem < 32) v &= (1u << rem) - 1u;
      w[q] = v;
    }
    return;
  }
  if (kind == QES_INIT_UP || kind == QES_INIT_DOWN) {
    for (int q = 0; q < nw; ++q) {
      uint32_t v = (kind == QES_INIT_UP) ? 0xffffffffu : 0u;
      const int rem = ns - 32 * q;
      if (rem < 32) v &= (1u << rem) - 1u;
      w[q] = v;
    }
    return;
  }
  // RND_FIXED: n_up ones at the front, then a Fisher-Yates shuffle driven by
  // counter (chain, pos, 0, 2).  Works on the packed words directly.
  for (int q = 0; q < nw; ++q) w[q] = 0u;
  for (int i = 0; i < n_up; ++i) w[i >> 5] |= 1u << (i & 31);
  for (int pos = ns - 1; pos > 0; --pos) {
    Philox4 r = philox4x32_10(cid, (uint32_t)pos, 0u, QES_STREAM_INIT_FIXED, k0, k1);
    const int j = (int)bounded_u32(r.x, (uint32_t)(pos + 1));
    const uint32_t bp = (w[pos >> 5] >> (pos & 31)) & 1u;
    const uint32_t bj = (w[j >> 5] >> (j & 31)) & 1u;
    if (bp != bj) {
      w[pos >> 5] ^= 1u << (pos & 31);
      w[j >> 5] ^= 1u << (j & 31);
    }
  }
}

extern "C" int qes_init_chains(int kind, int n_up, uint64_t seed, int64_t chain_offset, int n_chains, int ns,
                               uint32_t* bits_out, void* stream) {
  QES_ARG_CHECK(ns > 0 && n_chains >= 0 && bits_out != nullptr, "qes_init_chains: bad sizes/pointers");
  QES_ARG_CHECK(kind >= QES_INIT_RND && kind <= QES_INIT_DOWN, "qes_init_chains: unknown kind");
  QES_ARG_CHECK(kind != QES_INIT_RND_FIXED || (n_up >= 0 && n_up <= ns), "qes_init_chains: n_up out of range");
  if (n_chains == 0) return QES_OK;
  const int bs = 128;
  init_chains_kernel<<<(n_chains + bs - 1) / bs, bs, 0, (cudaStream_t)stream>>>(
      kind, n_up, (uint32_t)(seed & 0xffffffffu), (uint32_t)(seed >> 32), chain_offset, n_chains, ns, bits_out);
  QES_LAUNCH_CHECK();
  return QES_OK;
}

// ----------------------------------------------------------------------------
// ratio tables
// ----------------------------------------------------------------------------
QES_D void cosh_sinh2(float d, float& c, float& s) {
  const float e = expf(2.f * d), ei = 1.f / e;
  c = 0.5f * (e + ei);
  s = 0.5f * (e - ei);
}
QES_D void cosh_sinh2(float2 d, float2& c, float2& s) {
  // cosh(x+iy) = cosh x cos y + i sinh x sin y ; sinh(x+iy) = sinh x cos y + i cosh x sin y
  const float x = 2.f * d.x, y = 2.f * d.y;
  const float e = expf(x), ei = 1.f / e;
  const float ch = 0.5f * (e + ei), sh = 0.5f * (e - ei);
  float sn, cs;
  sincosf(y, &sn, &cs);
  c = make_float2(ch * cs, sh * sn);
  s = make_float2(sh * cs, ch * sn);
}

template <class T>
__global__ void move_tables_kernel(int nh, const T* __restrict__ a, const T* __restrict__ W, int K,
                                   const int32_t* __restrict__ mi, const int32_t* __restrict__ mj,
                                   const int32_t* __restrict__ mk, int move_major, T* __restrict__ Ct,
                                   T* __restrict__ St, T* __restrict__ A) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t total = (int64_t)K * nh;
  if (idx >= total) return;
  // layout [m][k] (local energy) or [k][m] (sampler)
  const int m = move_major ? (int)(idx % nh) : (int)(idx / K);
  const int k = move_major ? (int)(idx / nh) : (int)(idx % K);
  const int i = mi[k], j = mj[k], kind = mk[k];
  T d;
  if (kind == QES_MOVE_FLIP1) d = W[(int64_t)i * nh + m];
  else if (kind == QES_MOVE_PAIR_ANTI) d = addx(W[(int64_t)i * nh + m], scal(-1.f, W[(int64_t)j * nh + m]));
  else d = addx(W[(int64_t)i * nh + m], W[(int64_t)j * nh + m]);
  T c, s;
  cosh_sinh2(d, c, s);
  Ct[idx] = c;
  St[idx] = s;
  if (m == 0) {
    T av = a[i];
    if (kind == QES_MOVE_PAIR_ANTI) av = addx(av, scal(-1.f, a[j]));
    else if (kind == QES_MOVE_PAIR_PAR) av = addx(av, a[j]);
    A[k] = av;
  }
}

extern "C" int qes_rbm_move_tables(int dtype, int ns, int nh, const void* a, const void* W, int n_moves,
                                   const int32_t* move_i, const int32_t* move_j, const int32_t* move_kind,
                                   int move_major, void* Ct, void* St, void* A, void* stream) {
  QES_ARG_CHECK(ns > 0 && nh > 0 && n_moves >= 0, "qes_rbm_move_tables: bad sizes");
  QES_ARG_CHECK(dtype == QES_DTYPE_F32 || dtype == QES_DTYPE_C64, "qes_rbm_move_tables: bad dtype");
  if (n_moves == 0) return QES_OK;
  QES_ARG_CHECK(a && W && move_i && move_j && move_kind && Ct && St && A, "qes_rbm_move_tables: null pointer");
  const int64_t total = (int64_t)n_moves * nh;
  const int bs = 256;
  const unsigned grid = (unsigned)((total + bs - 1) / bs);
  if (dtype == QES_DTYPE_F32)
    move_tables_kernel<float><<<grid, bs, 0, (cudaStream_t)stream>>>(
        nh, (const float*)a, (const float*)W, n_moves, move_i, move_j, move_kind, move_major, (float*)Ct, (float*)St,
        (float*)A);
  else
    move_tables_kernel<float2><<<grid, bs, 0, (cudaStream_t)stream>>>(
        nh, (const float2*)a, (const float2*)W, n_moves, move_i, move_j, move_kind, move_major, (float2*)Ct,
        (float2*)St, (float2*)A);
  QES_LAUNCH_CHECK();
  return QES_OK;
}

// ----------------------------------------------------------------------------
// forward: theta, tanh(theta), log psi
// ----------------------------------------------------------------------------
// Block = SB samples; thread t owns hidden units m = t, t + blockDim, ...
// W is read once per block (coalesced across m); the signs come from the
// packed words staged in shared memory.
constexpr int FWD_SB = 16;
constexpr int FWD_THREADS = 256;

// One block of FWD_SB samples starting at row s0 (smem_words: FWD_SB * n_words(ns) words).
template <class T>
QES_D void rbm_forward_block(int64_t s0, uint32_t* smem_words, int ns, int nh, int64_t n_samples,
                             const uint32_t* __restrict__ bits, const T* __restrict__ a, const T* __restrict__ b,
                             const T* __restrict__ W, T* __restrict__ theta_out, T* __restrict__ tanh_out,
                             T* __restrict__ logpsi_out) {
  const int nw = n_words(ns);
  const int nsb = (int)min((int64_t)FWD_SB, n_samples - s0);
  for (int q = threadIdx.x; q < FWD_SB * nw; q += blockDim.x) {
    const int sl = q / nw;
    smem_words[q] = (sl < nsb) ? bits[(s0 + sl) * nw + (q % nw)] : 0u;
  }
  __syncthreads();

  T lsum[FWD_SB];
#pragma unroll
  for (int q = 0; q < FWD_SB; ++q) lsum[q] = ScalarTraits<T>::zero();

  for (int m = threadIdx.x; m < nh; m += blockDim.x) {
    T acc[FWD_SB];
    const T bm = b[m];
#pragma unroll
    for (int q = 0; q < FWD_SB; ++q) acc[q] = bm;
    for (int i = 0; i < ns; ++i) {
      const T w = W[(int64_t)i * nh + m];
#pragma unroll
      for (int q = 0; q < FWD_SB; ++q) {
        const uint32_t bit = (smem_words[q * nw + (i >> 5)] >> (i & 31)) & 1u;
        acc[q] = addx(acc[q], bit ? w : scal(-1.f, w));
      }
    }
#pragma unroll
    for (int q = 0; q < FWD_SB; ++q) {
      if (q < nsb) {
        const int64_t o = (s0 + q) * nh + m;
        if (theta_out) theta_out[o] = acc[q];
        if (tanh_out) tanh_out[o] = tanhx(acc[q]);
        lsum[q] = addx(lsum[q], log_cosh(acc[q]));
      }
    }
  }
  if (!logpsi_out) return;
  // visible term: thread t handles sites i = t, t + blockDim, ...
  for (int i = threadIdx.x; i < ns; i += blockDim.x) {
    const T ai = a[i];
#pragma unroll
    for (int q = 0; q < FWD_SB; ++q) {
      const uint32_t bit = (smem_words[q * nw + (i >> 5)] >> (i & 31)) & 1u;
      lsum[q] = addx(lsum[q], bit ? ai : scal(-1.f, ai));
    }
  }
  __shared__ T red[FWD_THREADS / 32][FWD_SB];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < FWD_SB; ++q) {
    T v = warp_sum(lsum[q]);
    if (lane == 0) red[warp][q] = v;
  }
  __syncthreads();
  if (threadIdx.x < FWD_SB && threadIdx.x < nsb) {
    T v = ScalarTraits<T>::zero();
    for (int w = 0; w < FWD_THREADS / 32; ++w) v = addx(v, red[w][threadIdx.x]);
    logpsi_out[s0 + threadIdx.x] = v;
  }
}

template <class T>
__global__ void __launch_bounds__(FWD_THREADS) rbm_forward_kernel(
    int ns, int nh, int64_t n_samples, const uint32_t* __restrict__ bits, const T* __restrict__ a,
    const T* __restrict__ b, const T* __restrict__ W, T* __restrict__ theta_out, T* __restrict__ tanh_out,
    T* __restrict__ logpsi_out) {
  extern __shared__ uint32_t smem_words[];
  rbm_forward_block<T>((int64_t)blockIdx.x * FWD_SB, smem_words, ns, nh, n_samples, bits, a, b, W, theta_out,
                       tanh_out, logpsi_out);
}

extern "C" int qes_rbm_forward(int dtype, int ns, int nh, int64_t n_samples, const uint32_t* bits, const void* a,
                               const void* b, const void* W, void* theta_out, void* tanh_out, void* logpsi_out,
                               void* stream) {
  QES_ARG_CHECK(ns > 0 && nh > 0 && n_samples >= 0, "qes_rbm_forward: bad sizes");
  QES_ARG_CHECK(dtype == QES_DTYPE_F32 || dtype == QES_DTYPE_C64, "qes_rbm_forward: bad dtype");
  QES_ARG_CHECK(bits && a && b && W, "qes_rbm_forward: null input");
  if (n_samples == 0) return QES_OK;
  const int nw = n_words(ns);
  const size_t sm = (size_t)FWD_SB * nw * sizeof(uint32_t);
  QES_ARG_CHECK(sm <= 48 * 1024, "qes_rbm_forward: ns too large");
  const unsigned grid = (unsigned)((n_samples + FWD_SB - 1) / FWD_SB);
  if (dtype == QES_DTYPE_F32)
    rbm_forward_kernel<float><<<grid, FWD_THREADS, sm, (cudaStream_t)stream>>>(
        ns, nh, n_samples, bits, (const float*)a, (const float*)b, (const float*)W, (float*)theta_out,
        (float*)tanh_out, (float*)logpsi_out);
  else
    rbm_forward_kernel<float2><<<grid, FWD_THREADS, sm, (cudaStream_t)stream>>>(
        ns, nh, n_samples, bits, (const float2*)a, (const float2*)b, (const float2*)W, (float2*)theta_out,
        (float2*)tanh_out, (float2*)logpsi_out);
  QES_LAUNCH_CHECK();
  return QES_OK;
}

// ----------------------------------------------------------------------------
// log-derivatives O (row-major, leading dimension ldo)
// ----------------------------------------------------------------------------
template <class T>
__global__ void log_derivatives_kernel(int ns, int nh, int64_t n_samples, const uint32_t* __restrict__ bits,
                                       const T* __restrict__ tanh_theta, T* __restrict__ O, int64_t ldo) {
  const int64_t s = blockIdx.y;
  if (s >= n_samples) return;
  const int nw = n_words(ns);
  const uint32_t* w = bits + s * nw;
  const int64_t P = (int64_t)ns + nh + (int64_t)ns * nh;
  T* row = O + s * ldo;
  const T* t = tanh_theta + s * nh;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < P; k += (int64_t)gridDim.x * blockDim.x) {
    T v;
    if (k < ns) {
      v = scal(sigma_of(w, (int)k), ScalarTraits<T>::one());
    } else if (k < ns + nh) {
      v = t[k - ns];
    } else {
      const int64_t q = k - ns - nh;
      const int i = (int)(q / nh), m = (int)(q % nh);
      v = scal(sigma_of(w, i), t[m]);
    }
    row[k] = v;
  }
}

extern "C" int qes_rbm_log_derivatives(int dtype, int ns, int nh, int64_t n_samples, const uint32_t* bits,
                                       const void* tanh_theta, void* O_out, int64_t ldo, void* stream) {
  QES_ARG_CHECK(ns > 0 && nh > 0 && n_samples >= 0, "qes_rbm_log_derivatives: bad sizes");
  const int64_t P = (int64_t)ns + nh + (int64_t)ns * nh;
  QES_ARG_CHECK(ldo >= P, "qes_rbm_log_derivatives: ldo < P");
  if (n_samples == 0) return QES_OK;
  QES_ARG_CHECK(bits && tanh_theta && O_out, "qes_rbm_log_derivatives: null pointer");
  const int bs = 256;
  const unsigned gx = (unsigned)std::min<int64_t>((P + bs - 1) / bs, 64);
  // grid.y is limited to 65535 rows: launch in row chunks
  for (int64_t r0 = 0; r0 < n_samples; r0 += 65535) {
    const int64_t nr = std::min<int64_t>(65535, n_samples - r0);
    dim3 grid(gx, (unsigned)nr);
    const int nw = n_words(ns);
    if (dtype == QES_DTYPE_F32)
      log_derivatives_kernel<float><<<grid, bs, 0, (cudaStream_t)stream>>>(
          ns, nh, nr, bits + r0 * nw, (const float*)tanh_theta + r0 * nh, (float*)O_out + r0 * ldo, ldo);
    else
      log_derivatives_kernel<float2><<<grid, bs, 0, (cudaStream_t)stream>>>(
          ns, nh, nr, bits + r0 * nw, (const float2*)tanh_theta + r0 * nh, (float2*)O_out + r0 * ldo, ldo);
    QES_LAUNCH_CHECK();
  }
  return QES_OK;
}

// ----------------------------------------------------------------------------
// float64 parameter update  master += lr * x ; params = (float) master
// ----------------------------------------------------------------------------
__global__ void param_update_kernel(int64_t n, double lr, const double* __restrict__ x, double* __restrict__ master,
                                    float* __restrict__ params) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
    const double v = master[k] + lr * x[k];
    master[k] = v;
    params[k] = (float)v;
  }
}

extern "C" int qes_param_update(int dtype, int64_t n_params, double lr, const void* x, void* master, void* params,
                                void* stream) {
  QES_ARG_CHECK(n_params >= 0 && x && master && params, "qes_param_update: bad arguments");
  QES_ARG_CHECK(dtype == QES_DTYPE_F32 || dtype == QES_DTYPE_C64, "qes_param_update: bad dtype");
  const int64_t n = (dtype == QES_DTYPE_C64) ? 2 * n_params : n_params;   // interleaved re/im
  if (n == 0) return QES_OK;
  const int bs = 256;
  const unsigned grid = (unsigned)std::min<int64_t>((n + bs - 1) / bs, 4096);
  param_update_kernel<<<grid, bs, 0, (cudaStream_t)stream>>>(n, lr, (const double*)x, (double*)master,
                                                             (float*)params);
  QES_LAUNCH_CHECK();
  return QES_OK;
}

// ----------------------------------------------------------------------------
// Batched problems
// ----------------------------------------------------------------------------
constexpr int BMT_THREADS = 256;

// items (b, first element / BMT_THREADS): one thread per table element
template <class T>
__global__ void __launch_bounds__(BMT_THREADS) batch_move_tables_kernel(
    const qes_batch_instance* __restrict__ inst, int mode, const int4* __restrict__ items,
    const T* __restrict__ params, const int32_t* __restrict__ mi, const int32_t* __restrict__ mj,
    const int32_t* __restrict__ mk, T* __restrict__ Ct, T* __restrict__ St, T* __restrict__ A) {
  const int4 it = items[blockIdx.x];
  const qes_batch_instance I = inst[it.x];
  const int nh = I.nh;
  const T* a = params + I.param_off;
  const T* W = a + I.ns + nh;
  const int K = (mode == 0) ? I.ns : I.n_moves;
  const int64_t idx = (int64_t)it.y * BMT_THREADS + threadIdx.x;
  if (idx >= (int64_t)K * nh) return;
  int m, k, i, j, kind;
  if (mode == 0) {                       // single flips, move-major
    m = (int)(idx % nh); k = (int)(idx / nh);
    i = k; j = k; kind = QES_MOVE_FLIP1;
  } else {                               // lowered moves, m-major
    m = (int)(idx / K); k = (int)(idx % K);
    i = mi[I.move_off + k]; j = mj[I.move_off + k]; kind = mk[I.move_off + k];
  }
  T d;
  if (kind == QES_MOVE_FLIP1) d = W[(int64_t)i * nh + m];
  else if (kind == QES_MOVE_PAIR_ANTI) d = addx(W[(int64_t)i * nh + m], scal(-1.f, W[(int64_t)j * nh + m]));
  else d = addx(W[(int64_t)i * nh + m], W[(int64_t)j * nh + m]);
  T c, s;
  cosh_sinh2(d, c, s);
  const int64_t off = (mode == 0) ? I.flip_off : I.move_table_off;
  Ct[off + idx] = c;
  St[off + idx] = s;
  if (mode == 1 && m == 0 && A) {
    T av = a[i];
    if (kind == QES_MOVE_PAIR_ANTI) av = addx(av, scal(-1.f, a[j]));
    else if (kind == QES_MOVE_PAIR_PAR) av = addx(av, a[j]);
    A[I.move_off + k] = av;
  }
}

extern "C" int qes_batch_move_tables(int dtype, int n_inst, const qes_batch_instance* inst, int mode, int n_items,
                                     const int32_t* items, const void* params, const int32_t* move_i,
                                     const int32_t* move_j, const int32_t* move_kind, void* Ct, void* St, void* A,
                                     void* stream) {
  QES_ARG_CHECK(dtype == QES_DTYPE_F32 || dtype == QES_DTYPE_C64, "qes_batch_move_tables: bad dtype");
  QES_ARG_CHECK(mode == 0 || mode == 1, "qes_batch_move_tables: mode must be 0 (flips) or 1 (moves)");
  QES_ARG_CHECK(n_inst >= 0 && n_items >= 0, "qes_batch_move_tables: bad sizes");
  if (n_items == 0) return QES_OK;
  QES_ARG_CHECK(inst && items && params && Ct && St, "qes_batch_move_tables: null pointer");
  QES_ARG_CHECK(mode == 0 || (move_i && move_j && move_kind && A), "qes_batch_move_tables: null move arrays");
  cudaStream_t st = (cudaStream_t)stream;
  if (dtype == QES_DTYPE_F32)
    batch_move_tables_kernel<float><<<n_items, BMT_THREADS, 0, st>>>(inst, mode, (const int4*)items,
                                                                     (const float*)params, move_i, move_j, move_kind,
                                                                     (float*)Ct, (float*)St, (float*)A);
  else
    batch_move_tables_kernel<float2><<<n_items, BMT_THREADS, 0, st>>>(inst, mode, (const int4*)items,
                                                                      (const float2*)params, move_i, move_j,
                                                                      move_kind, (float2*)Ct, (float2*)St,
                                                                      (float2*)A);
  QES_LAUNCH_CHECK();
  return QES_OK;
}

// items (b, sample block of FWD_SB)
template <class T>
__global__ void __launch_bounds__(FWD_THREADS) batch_forward_kernel(const qes_batch_instance* __restrict__ inst,
                                                                   const int4* __restrict__ items,
                                                                   const T* __restrict__ params,
                                                                   const uint32_t* __restrict__ bits,
                                                                   T* __restrict__ tanh_out, T* __restrict__ logpsi_out) {
  extern __shared__ uint32_t smem_words[];
  const int4 it = items[blockIdx.x];
  const qes_batch_instance I = inst[it.x];
  const T* a = params + I.param_off;
  const T* b = a + I.ns;
  const T* W = b + I.nh;
  const int64_t rows = (int64_t)I.n_chains * I.num_samples;
  rbm_forward_block<T>((int64_t)it.y * FWD_SB, smem_words, I.ns, I.nh, rows, bits + I.sample_word_off, a, b, W,
                       nullptr, tanh_out ? tanh_out + I.tanh_off : nullptr,
                       logpsi_out ? logpsi_out + I.sample_off : nullptr);
}

extern "C" int qes_batch_rbm_forward(int dtype, int n_inst, const qes_batch_instance* inst, int n_items,
                                     const int32_t* items, const void* params, const uint32_t* sample_bits,
                                     void* tanh_out, void* logpsi_out, void* stream) {
  QES_ARG_CHECK(dtype == QES_DTYPE_F32 || dtype == QES_DTYPE_C64, "qes_batch_rbm_forward: bad dtype");
  QES_ARG_CHECK(n_inst >= 0 && n_items >= 0, "qes_batch_rbm_forward: bad sizes");
  if (n_items == 0) return QES_OK;
  QES_ARG_CHECK(inst && items && params && sample_bits, "qes_batch_rbm_forward: null pointer");
  const size_t sm = (size_t)FWD_SB * 64 * sizeof(uint32_t);      // ns <= 2048
  cudaStream_t st = (cudaStream_t)stream;
  if (dtype == QES_DTYPE_F32)
    batch_forward_kernel<float><<<n_items, FWD_THREADS, sm, st>>>(inst, (const int4*)items, (const float*)params,
                                                                  sample_bits, (float*)tanh_out, (float*)logpsi_out);
  else
    batch_forward_kernel<float2><<<n_items, FWD_THREADS, sm, st>>>(inst, (const int4*)items, (const float2*)params,
                                                                   sample_bits, (float2*)tanh_out,
                                                                   (float2*)logpsi_out);
  QES_LAUNCH_CHECK();
  return QES_OK;
}

// ----------------------------------------------------------------------------
// replica swap of a region (Renyi-2 estimator): out_a takes region A from b and
// the rest from a, out_b the opposite (QES/NQS/src/nqs_entropy.py:311-460)
// ----------------------------------------------------------------------------
__global__ void swap_region_kernel(int64_t n_words_total, int nw, const uint32_t* __restrict__ mask,
                                   const uint32_t* __restrict__ a, const uint32_t* __restrict__ b,
                                   uint32_t* __restrict__ oa, uint32_t* __restrict__ ob) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n_words_total;
       k += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t m = mask[k % nw], x = a[k], y = b[k];
    oa[k] = (x & ~m) | (y & m);
    ob[k] = (y & ~m) | (x & m);
  }
}

extern "C" int qes_swap_region(int64_t n_samples, int ns, const uint32_t* mask_words, const uint32_t* bits_a,
                               const uint32_t* bits_b, uint32_t* out_a, uint32_t* out_b, void* stream) {
  QES_ARG_CHECK(n_samples >= 0 && ns > 0, "qes_swap_region: bad sizes");
  if (n_samples == 0) return QES_OK;
  QES_ARG_CHECK(mask_words && bits_a && bits_b && out_a && out_b, "qes_swap_region: null pointer");
  const int nw = n_words(ns);
  const int64_t total = n_samples * nw;
  const int bs = 256;
  const unsigned grid = (unsigned)std::min<int64_t>((total + bs - 1) / bs, 148 * 16);
  swap_region_kernel<<<grid, bs, 0, (cudaStream_t)stream>>>(total, nw, mask_words, bits_a, bits_b, out_a, out_b);
  QES_LAUNCH_CHECK();
  return QES_OK;
}
