// Exact ground energy by Lanczos on the GPU, matrix-free over the full S^z
// product basis (2^ns states, ns <= 32), from the same lowered Hamiltonian the
// local-energy kernel reads.
//
// Basis index: bit i of the index is site i (1 = up), the packed-spin
// convention of the library.  H acts as
//   (H x)(s) = diag(s) x(s) + sum_k active_k(s) conj(c_k(s)) x(s'_k),
// i.e. the matrix whose row s is the local energy's connected list (the
// estimator E_loc(s) = sum_k conj(c_k) psi(s')/psi(s) is <s|H|psi>/<s|psi>).
// Only Hamiltonians with real matrix elements are accepted (TFIM, XXZ, J1-J2
// all are: the sigma^y sigma^y slot has real coefficient -1/4 sigma_i sigma_j).
//
// Lanczos without re-orthogonalisation: the lowest Ritz value converges to the
// ground energy (spurious copies only duplicate converged values).  The
// tridiagonal eigenvalue is found by Sturm-sequence bisection in float64 on
// the host.  This replaces model.diagonalize(method='lanczos')
// (QES/Algebra/Hamil/hamil.py:1809+, hamil_diag_engine.py:176-305), whose
// eigen solver is not part of the reference snapshot.
#include "common.cuh"

#include <algorithm>
#include <cmath>
#include <map>
#include <vector>

#define QES_ARG_CHECK(cond, msg) do { if (!(cond)) { qes_set_last_message(msg); return QES_ERR_ARG; } } while (0)

constexpr int ED_THREADS = 256;
constexpr int ED_BLOCKS = 148 * 8;
constexpr int ED_MAX_TERMS = 512;      // per term kind, held in shared memory

struct EdTerms {
  int n_moves, n_zz, n_zf;
};

__global__ void __launch_bounds__(ED_THREADS) ed_matvec_kernel(
    int ns, EdTerms nt, const int32_t* __restrict__ mi, const int32_t* __restrict__ mj,
    const int32_t* __restrict__ mk, const float4* __restrict__ mcoef, const int32_t* __restrict__ zf_site,
    const float* __restrict__ zf_h, const int32_t* __restrict__ zz_i, const int32_t* __restrict__ zz_j,
    const float* __restrict__ zz_J, const double* __restrict__ x, double* __restrict__ y) {
  __shared__ uint64_t s_mask[ED_MAX_TERMS];    // bits flipped by move k
  __shared__ int2 s_ij[ED_MAX_TERMS];
  __shared__ int s_kind[ED_MAX_TERMS];
  __shared__ float2 s_c[ED_MAX_TERMS];          // real coefficient = c.x + sigma_i * c.y
  __shared__ int2 s_zz[ED_MAX_TERMS];
  __shared__ float s_zzJ[ED_MAX_TERMS];
  __shared__ int s_zf[ED_MAX_TERMS];
  __shared__ float s_zfh[ED_MAX_TERMS];
  for (int k = threadIdx.x; k < nt.n_moves; k += blockDim.x) {
    const int i = mi[k], j = mj[k], kind = mk[k];
    uint64_t m = 1ull << i;
    if (kind != QES_MOVE_FLIP1) m |= 1ull << j;
    s_mask[k] = m;
    s_ij[k] = make_int2(i, j);
    s_kind[k] = kind;
    const float4 c = mcoef[k];
    s_c[k] = make_float2(c.x, c.z);
  }
  for (int t = threadIdx.x; t < nt.n_zz; t += blockDim.x) { s_zz[t] = make_int2(zz_i[t], zz_j[t]); s_zzJ[t] = zz_J[t]; }
  for (int t = threadIdx.x; t < nt.n_zf; t += blockDim.x) { s_zf[t] = zf_site[t]; s_zfh[t] = zf_h[t]; }
  __syncthreads();
  const uint64_t dim = 1ull << ns;
  for (uint64_t s = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; s < dim; s += (uint64_t)gridDim.x * blockDim.x) {
    double d = 0.0;
    for (int t = 0; t < nt.n_zf; ++t) d += (double)s_zfh[t] * (((s >> s_zf[t]) & 1ull) ? 1.0 : -1.0);
    for (int t = 0; t < nt.n_zz; ++t) {
      const int2 p = s_zz[t];
      d += (double)s_zzJ[t] * ((((s >> p.x) ^ (s >> p.y)) & 1ull) ? -1.0 : 1.0);
    }
    double acc = d * x[s];
    for (int k = 0; k < nt.n_moves; ++k) {
      const int2 p = s_ij[k];
      const uint64_t bi = (s >> p.x) & 1ull;
      const int kind = s_kind[k];
      if (kind == QES_MOVE_PAIR_ANTI && bi == ((s >> p.y) & 1ull)) continue;
      if (kind == QES_MOVE_PAIR_PAR && bi != ((s >> p.y) & 1ull)) continue;
      const double c = (double)s_c[k].x + (bi ? 1.0 : -1.0) * (double)s_c[k].y;
      acc += c * x[s ^ s_mask[k]];
    }
    y[s] = acc;
  }
}

// partial dot products a.b per block
__global__ void __launch_bounds__(ED_THREADS) ed_dot_kernel(uint64_t n, const double* __restrict__ a,
                                                            const double* __restrict__ b, double* __restrict__ part) {
  double v = 0.0;
  for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (uint64_t)gridDim.x * blockDim.x)
    v += a[k] * b[k];
  __shared__ double red[ED_THREADS / 32];
  v = warp_sum(v);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int q = 0; q < ED_THREADS / 32; ++q) t += red[q];
    part[blockIdx.x] = t;
  }
}

// w = w - alpha v - beta v_prev, partial ||w||^2
__global__ void __launch_bounds__(ED_THREADS) ed_axpy_norm_kernel(uint64_t n, double alpha, double beta,
                                                                  const double* __restrict__ v,
                                                                  const double* __restrict__ vp, double* __restrict__ w,
                                                                  double* __restrict__ part) {
  double q2 = 0.0;
  for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (uint64_t)gridDim.x * blockDim.x) {
    const double t = w[k] - alpha * v[k] - beta * vp[k];
    w[k] = t;
    q2 += t * t;
  }
  __shared__ double red[ED_THREADS / 32];
  q2 = warp_sum(q2);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = q2;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int q = 0; q < ED_THREADS / 32; ++q) t += red[q];
    part[blockIdx.x] = t;
  }
}

// v_prev <- v ; v <- w / beta
__global__ void ed_shift_kernel(uint64_t n, double inv_beta, double* __restrict__ vp, double* __restrict__ v,
                                const double* __restrict__ w) {
  for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (uint64_t)gridDim.x * blockDim.x) {
    vp[k] = v[k];
    v[k] = w[k] * inv_beta;
  }
}

// random start vector (Philox, uniform in (-0.5, 0.5)), v_prev = 0, partial ||v||^2
__global__ void __launch_bounds__(ED_THREADS) ed_init_kernel(uint64_t n, uint32_t k0, uint32_t k1, double* __restrict__ v,
                                                             double* __restrict__ vp, double* __restrict__ part) {
  double q2 = 0.0;
  for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (uint64_t)gridDim.x * blockDim.x) {
    const Philox4 r = philox4x32_10((uint32_t)k, (uint32_t)(k >> 32), 0u, 3u, k0, k1);
    const double t = (double)uniform_open(r.x) - 0.5;
    v[k] = t;
    vp[k] = 0.0;
    q2 += t * t;
  }
  __shared__ double red[ED_THREADS / 32];
  q2 = warp_sum(q2);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = q2;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int q = 0; q < ED_THREADS / 32; ++q) t += red[q];
    part[blockIdx.x] = t;
  }
}

__global__ void ed_scale_kernel(uint64_t n, double s, double* __restrict__ v) {
  for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (uint64_t)gridDim.x * blockDim.x)
    v[k] *= s;
}

// number of eigenvalues of the symmetric tridiagonal (a, b) below x (Sturm sequence)
static int sturm_count(const std::vector<double>& a, const std::vector<double>& b, double x) {
  int cnt = 0;
  double q = 1.0;
  for (size_t i = 0; i < a.size(); ++i) {
    const double bb = (i == 0) ? 0.0 : b[i - 1] * b[i - 1];
    q = (a[i] - x) - (i == 0 ? 0.0 : bb / q);
    if (q == 0.0) q = -1e-300;
    if (q < 0.0) ++cnt;
  }
  return cnt;
}

static double tridiag_lowest(const std::vector<double>& a, const std::vector<double>& b) {
  double lo = a[0], hi = a[0];
  for (size_t i = 0; i < a.size(); ++i) {
    const double r = (i > 0 ? fabs(b[i - 1]) : 0.0) + (i + 1 < a.size() ? fabs(b[i]) : 0.0);
    lo = std::min(lo, a[i] - r);
    hi = std::max(hi, a[i] + r);
  }
  for (int it = 0; it < 200 && hi - lo > 1e-15 * std::max(1.0, fabs(lo)); ++it) {
    const double mid = 0.5 * (lo + hi);
    if (sturm_count(a, b, mid) >= 1) hi = mid;
    else lo = mid;
  }
  return 0.5 * (lo + hi);
}

static int ed_sum(const double* dpart, double* hpart, cudaStream_t st, double* out) {
  QES_CUDA_CHECK(cudaMemcpyAsync(hpart, dpart, ED_BLOCKS * sizeof(double), cudaMemcpyDeviceToHost, st));
  QES_CUDA_CHECK(cudaStreamSynchronize(st));
  double s = 0.0;
  for (int q = 0; q < ED_BLOCKS; ++q) s += hpart[q];
  *out = s;
  return QES_OK;
}

// Lanczos three-term recursion on the caller's vectors (v, vp, w of n float64 each, part of
// ED_BLOCKS partial sums); matvec(x, y) launches y = H x on st.  Stops when the lowest Ritz value
// changes by <= tol * max(1, |E|) after the eighth iteration or the Krylov space is exhausted.
template <class Matvec>
static int ed_lanczos_loop(uint64_t n, Matvec&& matvec, double* v, double* vp, double* w, double* part, int max_iter,
                           double tol, uint64_t seed, cudaStream_t st, double* e0_out, int* iterations_out) {
  int rc = QES_OK;
  std::vector<double> hpart(ED_BLOCKS), alpha, beta;
  ed_init_kernel<<<ED_BLOCKS, ED_THREADS, 0, st>>>(n, (uint32_t)seed, (uint32_t)(seed >> 32), v, vp, part);
  QES_LAUNCH_CHECK();
  double nrm2 = 0.0;
  if ((rc = ed_sum(part, hpart.data(), st, &nrm2))) return rc;
  ed_scale_kernel<<<ED_BLOCKS, ED_THREADS, 0, st>>>(n, 1.0 / sqrt(nrm2), v);
  QES_LAUNCH_CHECK();
  double e_prev = 0.0, e = 0.0, b_prev = 0.0;
  int it = 0;
  bool conv = false;
  for (; it < max_iter; ++it) {
    matvec(v, w);
    ed_dot_kernel<<<ED_BLOCKS, ED_THREADS, 0, st>>>(n, v, w, part);
    QES_LAUNCH_CHECK_N(2);
    double a = 0.0;
    if ((rc = ed_sum(part, hpart.data(), st, &a))) return rc;
    alpha.push_back(a);
    ed_axpy_norm_kernel<<<ED_BLOCKS, ED_THREADS, 0, st>>>(n, a, b_prev, v, vp, w, part);
    QES_LAUNCH_CHECK();
    double b2 = 0.0;
    if ((rc = ed_sum(part, hpart.data(), st, &b2))) return rc;
    const double b = sqrt(b2);
    e = tridiag_lowest(alpha, beta);
    if ((it >= 8 && fabs(e - e_prev) <= tol * std::max(1.0, fabs(e))) || b <= 1e-12 * std::max(1.0, fabs(e))) {
      conv = true;
      ++it;
      break;
    }
    e_prev = e;
    beta.push_back(b);
    ed_shift_kernel<<<ED_BLOCKS, ED_THREADS, 0, st>>>(n, 1.0 / b, vp, v, w);
    QES_LAUNCH_CHECK();
    b_prev = b;
  }
  *e0_out = e;
  if (iterations_out) *iterations_out = it;
  return conv ? QES_OK : QES_ERR_NOT_CONVERGED;
}

static int ed_check(int ns, const qes_hamiltonian* ham) {
  QES_ARG_CHECK(ns > 0 && ns <= 32 && ham != nullptr, "qes_ed: need 0 < ns <= 32");
  QES_ARG_CHECK(ham->n_moves >= 0 && ham->n_moves <= ED_MAX_TERMS && ham->n_zz <= ED_MAX_TERMS &&
                    ham->n_zfield <= ED_MAX_TERMS,
                "qes_ed: too many terms");
  QES_ARG_CHECK(ham->n_moves == 0 || (ham->move_i && ham->move_j && ham->move_kind && ham->move_coef),
                "qes_ed: null move arrays");
  return QES_OK;
}

static void ed_launch_matvec(int ns, const qes_hamiltonian* ham, const double* x, double* y, cudaStream_t st) {
  EdTerms nt{ham->n_moves, ham->n_zz, ham->n_zfield};
  ed_matvec_kernel<<<ED_BLOCKS, ED_THREADS, 0, st>>>(ns, nt, ham->move_i, ham->move_j, ham->move_kind,
                                                     (const float4*)ham->move_coef, ham->zf_site, ham->zf_h, ham->zz_i,
                                                     ham->zz_j, ham->zz_J, x, y);
}

extern "C" int qes_ed_matvec(int ns, const qes_hamiltonian* ham, const double* x, double* y, void* stream) {
  int rc = ed_check(ns, ham);
  if (rc) return rc;
  QES_ARG_CHECK(x && y, "qes_ed_matvec: null vector");
  ed_launch_matvec(ns, ham, x, y, (cudaStream_t)stream);
  QES_LAUNCH_CHECK();
  return QES_OK;
}

extern "C" int qes_ed_workspace_bytes(int ns, size_t* bytes) {
  QES_ARG_CHECK(bytes && ns > 0 && ns <= 32, "qes_ed_workspace_bytes: need 0 < ns <= 32");
  *bytes = 3 * ((size_t)8 << ns) + ED_BLOCKS * sizeof(double);
  return QES_OK;
}

extern "C" int qes_ed_lanczos(int ns, const qes_hamiltonian* ham, int max_iter, double tol, uint64_t seed,
                              double* e0_out, int* iterations_out, void* workspace, size_t workspace_bytes,
                              void* stream) {
  int rc = ed_check(ns, ham);
  if (rc) return rc;
  QES_ARG_CHECK(e0_out && max_iter >= 2 && tol > 0.0, "qes_ed_lanczos: bad args");
  size_t need = 0;
  qes_ed_workspace_bytes(ns, &need);
  if (!workspace || workspace_bytes < need) {
    qes_set_last_message("qes_ed_lanczos: workspace too small");
    return QES_ERR_WORKSPACE;
  }
  // the matrix elements must be real: coefficient imaginary parts are zero
  if (ham->n_moves > 0) {
    std::vector<float> c((size_t)ham->n_moves * 4);
    cudaStream_t st0 = (cudaStream_t)stream;
    QES_CUDA_CHECK(cudaMemcpyAsync(c.data(), ham->move_coef, c.size() * sizeof(float), cudaMemcpyDeviceToHost, st0));
    QES_CUDA_CHECK(cudaStreamSynchronize(st0));
    for (int k = 0; k < ham->n_moves; ++k)
      QES_ARG_CHECK(c[4 * k + 1] == 0.f && c[4 * k + 3] == 0.f, "qes_ed_lanczos: complex matrix elements");
  }
  const uint64_t n = 1ull << ns;
  cudaStream_t st = (cudaStream_t)stream;
  double* v = (double*)workspace;
  double* vp = v + n;
  double* w = vp + n;
  double* part = w + n;
  auto matvec = [&](const double* x, double* y) { ed_launch_matvec(ns, ham, x, y, st); };
  return ed_lanczos_loop(n, matvec, v, vp, w, part, max_iter, tol, seed, st, e0_out, iterations_out);
}

// ================================================================================================
// S^z sector (and spin-flip parity) Lanczos
// ================================================================================================
// Basis: the states of ns sites with n_up up spins, indexed by their colex rank
//   rank(s) = sum_k C(p_k, k + 1),  p_0 < p_1 < ... the positions of the set bits,
// so that a state is found from its bits and back in O(n_up) with a binomial table (no lookup
// array).  With spin-flip parity (ns = 2 n_up, no z field) a state and its flip ~s are one
// basis vector; the representative is the one whose top site (ns - 1) is down, i.e. the
// n_up-subsets of the lower ns - 1 sites, and psi(~s) = parity * psi(s).  The Hamiltonian must
// conserve S^z: pair moves of anti-parallel spins only (no single flips, no pair flips of parallel
// spins, which the lowering drops for the isotropic models).
constexpr int ED_BINOM_N = 65, ED_BINOM_K = 33;

struct EdSector {
  int ns, n_up, bits;        // bits: ns, or ns - 1 with spin-flip parity (the representatives' range)
  int parity;                // 0: none, +1 / -1: spin-flip parity
};

__device__ __forceinline__ uint64_t ed_rank(uint64_t s, int n_up, const uint64_t* __restrict__ C) {
  uint64_t r = 0;
  for (int k = 0; k < n_up; ++k) {
    const int p = __ffsll((long long)s) - 1;
    r += C[p * ED_BINOM_K + k + 1];
    s &= s - 1;
  }
  return r;
}

__device__ __forceinline__ uint64_t ed_unrank(uint64_t r, int n_up, int bits, const uint64_t* __restrict__ C) {
  uint64_t s = 0;
  int p = bits - 1;
  for (int k = n_up; k >= 1; --k) {
    while (C[p * ED_BINOM_K + k] > r) --p;           // largest p with C(p, k) <= r
    r -= C[p * ED_BINOM_K + k];
    s |= 1ull << p;
    --p;
  }
  return s;
}

__global__ void __launch_bounds__(ED_THREADS) ed_sector_matvec_kernel(
    EdSector sec, uint64_t dim, EdTerms nt, const int32_t* __restrict__ mi, const int32_t* __restrict__ mj,
    const float4* __restrict__ mcoef, const int32_t* __restrict__ zf_site, const float* __restrict__ zf_h,
    const int32_t* __restrict__ zz_i, const int32_t* __restrict__ zz_j, const float* __restrict__ zz_J,
    const uint64_t* __restrict__ binom, const double* __restrict__ x, double* __restrict__ y) {
  __shared__ uint64_t C[ED_BINOM_N * ED_BINOM_K];
  __shared__ uint64_t s_mask[ED_MAX_TERMS];
  __shared__ int2 s_ij[ED_MAX_TERMS];
  __shared__ float s_c[ED_MAX_TERMS];
  __shared__ int2 s_zz[ED_MAX_TERMS];
  __shared__ float s_zzJ[ED_MAX_TERMS];
  __shared__ int s_zf[ED_MAX_TERMS];
  __shared__ float s_zfh[ED_MAX_TERMS];
  for (int t = threadIdx.x; t < ED_BINOM_N * ED_BINOM_K; t += blockDim.x) C[t] = binom[t];
  for (int k = threadIdx.x; k < nt.n_moves; k += blockDim.x) {
    const int i = mi[k], j = mj[k];
    s_mask[k] = (1ull << i) | (1ull << j);
    s_ij[k] = make_int2(i, j);
    s_c[k] = mcoef[k].x;
  }
  for (int t = threadIdx.x; t < nt.n_zz; t += blockDim.x) { s_zz[t] = make_int2(zz_i[t], zz_j[t]); s_zzJ[t] = zz_J[t]; }
  for (int t = threadIdx.x; t < nt.n_zf; t += blockDim.x) { s_zf[t] = zf_site[t]; s_zfh[t] = zf_h[t]; }
  __syncthreads();
  const uint64_t full = (sec.ns == 64) ? ~0ull : ((1ull << sec.ns) - 1ull);
  const uint64_t top = 1ull << (sec.ns - 1);
  for (uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; r < dim; r += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t s = ed_unrank(r, sec.n_up, sec.bits, C);
    double d = 0.0;
    for (int t = 0; t < nt.n_zf; ++t) d += (double)s_zfh[t] * (((s >> s_zf[t]) & 1ull) ? 1.0 : -1.0);
    for (int t = 0; t < nt.n_zz; ++t) {
      const int2 p = s_zz[t];
      d += (double)s_zzJ[t] * ((((s >> p.x) ^ (s >> p.y)) & 1ull) ? -1.0 : 1.0);
    }
    double acc = d * x[r];
    for (int k = 0; k < nt.n_moves; ++k) {
      const int2 p = s_ij[k];
      if (((s >> p.x) ^ (s >> p.y)) & 1ull) {           // anti-parallel: the exchange is allowed
        uint64_t t2 = s ^ s_mask[k];
        double f = (double)s_c[k];
        if (sec.parity != 0 && (t2 & top)) {             // back to the representative of {t2, ~t2}
          t2 = ~t2 & full;
          f *= (double)sec.parity;
        }
        acc += f * x[ed_rank(t2, sec.n_up, C)];
      }
    }
    y[r] = acc;
  }
}

namespace {
void ed_binomials(std::vector<uint64_t>& C) {
  C.assign((size_t)ED_BINOM_N * ED_BINOM_K, 0ull);
  for (int n = 0; n < ED_BINOM_N; ++n) {
    C[(size_t)n * ED_BINOM_K] = 1ull;
    for (int k = 1; k < ED_BINOM_K && k <= n; ++k)
      C[(size_t)n * ED_BINOM_K + k] = C[(size_t)(n - 1) * ED_BINOM_K + k - 1] +
                                       (k <= n - 1 ? C[(size_t)(n - 1) * ED_BINOM_K + k] : 0ull);
  }
}

int ed_sector_dims(int ns, int n_up, int parity, uint64_t* dim, EdSector* sec) {
  QES_ARG_CHECK(ns > 0 && ns <= 62 && n_up >= 0 && n_up <= ns && n_up < ED_BINOM_K,
                "qes_ed_sector: need 0 < ns <= 62 and n_up <= 32");
  QES_ARG_CHECK(parity == 0 || ((parity == 1 || parity == -1) && 2 * n_up == ns),
                "qes_ed_sector: spin-flip parity needs ns = 2 n_up");
  std::vector<uint64_t> C;
  ed_binomials(C);
  const int bits = parity ? ns - 1 : ns;
  *dim = C[(size_t)bits * ED_BINOM_K + n_up];
  if (sec) *sec = EdSector{ns, n_up, bits, parity};
  return QES_OK;
}
}  // namespace

extern "C" int qes_ed_sector_dim(int ns, int n_up, int parity, uint64_t* dim) {
  QES_ARG_CHECK(dim, "qes_ed_sector_dim: null output");
  return ed_sector_dims(ns, n_up, parity, dim, nullptr);
}

extern "C" int qes_ed_sector_workspace_bytes(int ns, int n_up, int parity, size_t* bytes) {
  QES_ARG_CHECK(bytes, "qes_ed_sector_workspace_bytes: null output");
  uint64_t dim = 0;
  int rc = ed_sector_dims(ns, n_up, parity, &dim, nullptr);
  if (rc) return rc;
  *bytes = 3 * (size_t)dim * sizeof(double) + ED_BLOCKS * sizeof(double) +
           (size_t)ED_BINOM_N * ED_BINOM_K * sizeof(uint64_t) + 256;
  return QES_OK;
}

extern "C" int qes_ed_lanczos_sector(int ns, int n_up, int parity, const qes_hamiltonian* ham, int max_iter,
                                     double tol, uint64_t seed, double* e0_out, int* iterations_out,
                                     void* workspace, size_t workspace_bytes, void* stream) {
  QES_ARG_CHECK(ham && e0_out && max_iter >= 2 && tol > 0.0, "qes_ed_lanczos_sector: bad args");
  QES_ARG_CHECK(ham->n_moves >= 0 && ham->n_moves <= ED_MAX_TERMS && ham->n_zz <= ED_MAX_TERMS &&
                    ham->n_zfield <= ED_MAX_TERMS,
                "qes_ed_lanczos_sector: too many terms");
  uint64_t dim = 0;
  EdSector sec{};
  int rc = ed_sector_dims(ns, n_up, parity, &dim, &sec);
  if (rc) return rc;
  QES_ARG_CHECK(dim >= 1, "qes_ed_lanczos_sector: empty sector");
  QES_ARG_CHECK(!(parity != 0 && ham->n_zfield > 0), "qes_ed_lanczos_sector: a z field breaks the spin-flip parity");
  size_t need = 0;
  qes_ed_sector_workspace_bytes(ns, n_up, parity, &need);
  if (!workspace || workspace_bytes < need) {
    qes_set_last_message("qes_ed_lanczos_sector: workspace too small");
    return QES_ERR_WORKSPACE;
  }
  cudaStream_t st = (cudaStream_t)stream;
  // S^z conservation and real matrix elements: anti-parallel pair moves only, real coefficients
  if (ham->n_moves > 0) {
    std::vector<float> c((size_t)ham->n_moves * 4);
    std::vector<int32_t> kind(ham->n_moves);
    QES_CUDA_CHECK(cudaMemcpyAsync(c.data(), ham->move_coef, c.size() * sizeof(float), cudaMemcpyDeviceToHost, st));
    QES_CUDA_CHECK(cudaMemcpyAsync(kind.data(), ham->move_kind, kind.size() * sizeof(int32_t), cudaMemcpyDeviceToHost,
                                   st));
    QES_CUDA_CHECK(cudaStreamSynchronize(st));
    for (int k = 0; k < ham->n_moves; ++k) {
      QES_ARG_CHECK(kind[k] == QES_MOVE_PAIR_ANTI, "qes_ed_lanczos_sector: the Hamiltonian does not conserve S^z");
      QES_ARG_CHECK(c[4 * k + 1] == 0.f && c[4 * k + 2] == 0.f && c[4 * k + 3] == 0.f,
                    "qes_ed_lanczos_sector: complex matrix elements");
    }
  }
  double* v = (double*)workspace;
  double* vp = v + dim;
  double* w = vp + dim;
  double* part = w + dim;
  uint64_t* binom = reinterpret_cast<uint64_t*>(part + ED_BLOCKS);
  std::vector<uint64_t> C;
  ed_binomials(C);
  QES_CUDA_CHECK(cudaMemcpyAsync(binom, C.data(), C.size() * sizeof(uint64_t), cudaMemcpyHostToDevice, st));
  const EdTerms nt{ham->n_moves, ham->n_zz, ham->n_zfield};
  auto matvec = [&](const double* x, double* y) {
    ed_sector_matvec_kernel<<<ED_BLOCKS, ED_THREADS, 0, st>>>(sec, dim, nt, ham->move_i, ham->move_j,
                                                              (const float4*)ham->move_coef, ham->zf_site, ham->zf_h,
                                                              ham->zz_i, ham->zz_j, ham->zz_J, binom, x, y);
  };
  rc = ed_lanczos_loop(dim, matvec, v, vp, w, part, max_iter, tol, seed, st, e0_out, iterations_out);
  // the binomial table was copied from a host vector: finish the stream before it goes out of scope
  QES_CUDA_CHECK(cudaStreamSynchronize(st));
  return rc;
}

// ================================================================================================
// Translation (and spin-flip) reduced S^z sector on an lx x ly torus
// ================================================================================================
// Group G: the lx*ly translations T(a, b): site (x, y) -> ((x + a) mod lx, (y + b) mod ly) (site
// index x + lx*y, a chain is ly = 1), times the spin flip F when parity != 0; M = |G|.  Its real
// one-dimensional representations are used: chi(T(a, b) F^f) = (-1)^(kx a + ky b) * parity^f with
// kx, ky in {0, 1}, i.e. momentum 0 or pi along each axis.  A representative r is the smallest
// state of its orbit O_r; the symmetric basis vector is
//   |r~> = |O_r|^-1/2 sum_{s in O_r} chi(h_s) |s>,   h_s r = s,
// and orbits on whose stabiliser chi is not 1 have no vector in the sector.  Since H commutes
// with G, the reduced matrix is
//   <r~|H|r'~> = sum_{s in O_r'} <s|H|r> chi(h_s) sqrt(|stab r'| / |stab r|),
// so row r visits the states s connected to r, maps each to its representative r' = g s (the
// transform g reaching the orbit minimum; chi(h_s) = chi(g) for a real character) and counts the
// transforms that reach it (|stab r'|).  Representatives are listed in increasing order (= colex
// rank order at a fixed number of up spins), in buckets of 32 ranks: off[b] .. off[b + 1] are
// the list positions of the representatives of rank 32 b .. 32 b + 31, so finding a state is
// one rank, two offsets and a scan of the few entries of its bucket.  The momentum sectors are
// those of QES/Algebra/Symmetries/translation.py:470-519 (character exp(2 pi i k n / L)) with
// k = 0 or L / 2, which keep the reduced matrix real; the spin flip is the parity of
// QES/Algebra/Symmetries/parity.py.
constexpr int ED_SCAN_PER_THREAD = 16;
constexpr int ED_SCAN_TILE = ED_THREADS * ED_SCAN_PER_THREAD;
constexpr uint64_t ED_SYMM_MAX_RANKS = 1ull << 37;   // the enumeration passes visit every rank

struct EdTorus {
  int lx, ly, ns, n_up, bits;   // bits: the rank space (ns - 1 with the flip: representatives have site ns - 1 down)
  int parity, kx, ky;
  uint64_t full, n_ranks, n_buckets, n_tiles;
};

struct EdTorusSmem {
  uint64_t C[ED_BINOM_N * ED_BINOM_K];
  uint64_t hi[64], lo[64];   // x translation by a: sites with x >= a receive bits from x - a, sites x < a from x - a + lx
};

__device__ __forceinline__ void ed_torus_tables(const EdTorus& T, const uint64_t* __restrict__ binom,
                                                EdTorusSmem& sm) {
  for (int t = threadIdx.x; t < ED_BINOM_N * ED_BINOM_K; t += blockDim.x) sm.C[t] = binom[t];
  for (int a = threadIdx.x; a < T.lx; a += blockDim.x) {
    const uint64_t row = (1ull << T.lx) - 1ull;
    const uint64_t below = (1ull << a) - 1ull;
    uint64_t h = 0, l = 0;
    for (int y = 0; y < T.ly; ++y) {
      h |= (row & ~below) << (y * T.lx);
      l |= below << (y * T.lx);
    }
    sm.hi[a] = h;
    sm.lo[a] = l;
  }
}

__device__ __forceinline__ uint64_t ed_shift_x(uint64_t r, int a, const EdTorus& T, const EdTorusSmem& sm) {
  return ((r << a) & sm.hi[a]) | ((r >> (T.lx - a)) & sm.lo[a]);
}

__device__ __forceinline__ uint64_t ed_shift_row(uint64_t r, const EdTorus& T) {
  return ((r << T.lx) | (r >> (T.ns - T.lx))) & T.full;
}

// s is a representative of the sector: no transform maps it below itself, and every transform that
// fixes it has character 1 (early exit at the first transform that fails)
__device__ __forceinline__ bool ed_is_rep(uint64_t s, const EdTorus& T, const EdTorusSmem& sm) {
  uint64_t r = s;
  for (int b = 0; b < T.ly; ++b) {
    for (int a = 0; a < T.lx; ++a) {
      const uint64_t t = ed_shift_x(r, a, T, sm);
      const int neg = ((T.kx & a) ^ (T.ky & b)) & 1;
      if (t < s || (t == s && neg)) return false;
      if (T.parity) {
        const uint64_t f = ~t & T.full;
        if (f < s || (f == s && (neg ^ (T.parity < 0)))) return false;
      }
    }
    r = ed_shift_row(r, T);
  }
  return true;
}

struct EdOrbit {
  uint64_t m;   // orbit minimum
  int stab;     // transforms reaching it (= |stabiliser|)
  int neg;      // their character is -1
  bool ok;      // all of them have the same character (else the orbit is not in the sector)
};

__device__ __forceinline__ void ed_orbit_take(EdOrbit& o, uint64_t t, int neg) {
  if (t < o.m) {
    o.m = t;
    o.stab = 1;
    o.neg = neg;
    o.ok = true;
  } else if (t == o.m) {
    ++o.stab;
    o.ok = o.ok && (neg == o.neg);
  }
}

__device__ __forceinline__ EdOrbit ed_orbit(uint64_t s, const EdTorus& T, const EdTorusSmem& sm) {
  EdOrbit o{~0ull, 0, 0, true};
  uint64_t r = s;
  for (int b = 0; b < T.ly; ++b) {
    for (int a = 0; a < T.lx; ++a) {
      const uint64_t t = ed_shift_x(r, a, T, sm);
      const int neg = ((T.kx & a) ^ (T.ky & b)) & 1;
      ed_orbit_take(o, t, neg);
      if (T.parity) ed_orbit_take(o, ~t & T.full, neg ^ (T.parity < 0));
    }
    r = ed_shift_row(r, T);
  }
  return o;
}

// list position of representative m, -1 when it is not listed
__device__ __forceinline__ int64_t ed_rep_index(uint64_t m, const EdTorus& T, const EdTorusSmem& sm,
                                                const uint32_t* __restrict__ off, const uint64_t* __restrict__ reps) {
  const uint64_t b = ed_rank(m, T.n_up, sm.C) >> 5;
  const uint32_t lo = off[b], hi = off[b + 1];
  for (uint32_t q = lo; q < hi; ++q)
    if (reps[q] == m) return (int64_t)q;
  return -1;
}

// Enumeration, pass 1: one warp per bucket of 32 ranks; cnt[b] = representatives in bucket b (when
// cnt is given) and per-block totals.
__global__ void __launch_bounds__(ED_THREADS) ed_symm_count_kernel(EdTorus T, const uint64_t* __restrict__ binom,
                                                                   uint32_t* __restrict__ cnt,
                                                                   unsigned long long* __restrict__ part) {
  __shared__ EdTorusSmem sm;
  __shared__ unsigned long long red[ED_THREADS / 32];
  ed_torus_tables(T, binom, sm);
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const uint64_t n_warps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  unsigned long long total = 0;
  for (uint64_t b = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; b < T.n_buckets; b += n_warps) {
    const uint64_t rk = b * 32 + lane;
    const bool is = rk < T.n_ranks && ed_is_rep(ed_unrank(rk, T.n_up, T.bits, sm.C), T, sm);
    const unsigned bal = __ballot_sync(~0u, is);
    if (lane == 0) {
      if (cnt) cnt[b] = (uint32_t)__popc(bal);
      total += (unsigned long long)__popc(bal);
    }
  }
  if (lane == 0) red[threadIdx.x >> 5] = total;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long t = 0;
    for (int q = 0; q < ED_THREADS / 32; ++q) t += red[q];
    part[blockIdx.x] = t;
  }
}

// Pass 2: sums of tiles of ED_SCAN_TILE bucket counts (one block per tile)
__global__ void __launch_bounds__(ED_THREADS) ed_tile_sum_kernel(uint64_t n, uint64_t n_tiles,
                                                                 const uint32_t* __restrict__ cnt,
                                                                 unsigned long long* __restrict__ tsum) {
  __shared__ unsigned long long red[ED_THREADS / 32];
  for (uint64_t tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
    const uint64_t base = tile * ED_SCAN_TILE;
    unsigned long long v = 0;
    for (int q = threadIdx.x; q < ED_SCAN_TILE; q += blockDim.x)
      if (base + q < n) v += cnt[base + q];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(~0u, v, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
      unsigned long long t = 0;
      for (int q = 0; q < ED_THREADS / 32; ++q) t += red[q];
      tsum[tile] = t;
    }
    __syncthreads();
  }
}

// Pass 3: bucket counts -> exclusive offsets in place (one block per tile, toff = the tiles'
// exclusive offsets); off[n] = total
__global__ void __launch_bounds__(ED_THREADS) ed_tile_scan_kernel(uint64_t n, uint64_t n_tiles, uint32_t* __restrict__ off,
                                                                  const unsigned long long* __restrict__ toff,
                                                                  uint64_t total) {
  __shared__ uint32_t wsum[ED_THREADS / 32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (uint64_t tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
    const uint64_t base = tile * ED_SCAN_TILE + (uint64_t)threadIdx.x * ED_SCAN_PER_THREAD;
    uint32_t v[ED_SCAN_PER_THREAD];
    uint32_t s = 0;
#pragma unroll
    for (int q = 0; q < ED_SCAN_PER_THREAD; ++q) {
      v[q] = (base + q < n) ? off[base + q] : 0u;
      s += v[q];
    }
    uint32_t inc = s;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t t = __shfl_up_sync(~0u, inc, o);
      if (lane >= o) inc += t;
    }
    if (lane == 31) wsum[wid] = inc;
    __syncthreads();
    uint32_t run = (uint32_t)toff[tile] + inc - s;
    for (int q = 0; q < wid; ++q) run += wsum[q];
#pragma unroll
    for (int q = 0; q < ED_SCAN_PER_THREAD; ++q) {
      if (base + q < n) off[base + q] = run;
      run += v[q];
    }
    __syncthreads();
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) off[n] = (uint32_t)total;
}

// Pass 4: the representatives in increasing order (one warp per bucket, as pass 1)
__global__ void __launch_bounds__(ED_THREADS) ed_symm_fill_kernel(EdTorus T, const uint64_t* __restrict__ binom,
                                                                  const uint32_t* __restrict__ off,
                                                                  uint64_t* __restrict__ reps) {
  __shared__ EdTorusSmem sm;
  ed_torus_tables(T, binom, sm);
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const uint64_t n_warps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t b = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; b < T.n_buckets; b += n_warps) {
    const uint64_t rk = b * 32 + lane;
    uint64_t s = 0;
    bool is = false;
    if (rk < T.n_ranks) {
      s = ed_unrank(rk, T.n_up, T.bits, sm.C);
      is = ed_is_rep(s, T, sm);
    }
    const unsigned bal = __ballot_sync(~0u, is);
    if (is) reps[off[b] + (uint32_t)__popc(bal & ((1u << lane) - 1u))] = s;
  }
}

// y = H x in the symmetric basis; one thread per representative.  missing counts connected
// representatives absent from the list (zero for a Hamiltonian that commutes with the group).
__global__ void __launch_bounds__(ED_THREADS) ed_symm_matvec_kernel(
    EdTorus T, uint64_t dim, EdTerms nt, const int32_t* __restrict__ mi, const int32_t* __restrict__ mj,
    const float4* __restrict__ mcoef, const int32_t* __restrict__ zf_site, const float* __restrict__ zf_h,
    const int32_t* __restrict__ zz_i, const int32_t* __restrict__ zz_j, const float* __restrict__ zz_J,
    const uint64_t* __restrict__ binom, const uint32_t* __restrict__ off, const uint64_t* __restrict__ reps,
    const double* __restrict__ x, double* __restrict__ y, unsigned long long* __restrict__ missing) {
  __shared__ EdTorusSmem sm;
  __shared__ uint64_t s_mask[ED_MAX_TERMS];
  __shared__ int2 s_ij[ED_MAX_TERMS];
  __shared__ float s_c[ED_MAX_TERMS];
  __shared__ int2 s_zz[ED_MAX_TERMS];
  __shared__ float s_zzJ[ED_MAX_TERMS];
  __shared__ int s_zf[ED_MAX_TERMS];
  __shared__ float s_zfh[ED_MAX_TERMS];
  ed_torus_tables(T, binom, sm);
  for (int k = threadIdx.x; k < nt.n_moves; k += blockDim.x) {
    const int i = mi[k], j = mj[k];
    s_mask[k] = (1ull << i) | (1ull << j);
    s_ij[k] = make_int2(i, j);
    s_c[k] = mcoef[k].x;
  }
  for (int t = threadIdx.x; t < nt.n_zz; t += blockDim.x) { s_zz[t] = make_int2(zz_i[t], zz_j[t]); s_zzJ[t] = zz_J[t]; }
  for (int t = threadIdx.x; t < nt.n_zf; t += blockDim.x) { s_zf[t] = zf_site[t]; s_zfh[t] = zf_h[t]; }
  __syncthreads();
  unsigned long long miss = 0;
  for (uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; r < dim; r += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t s = reps[r];
    const double inv_stab = 1.0 / (double)ed_orbit(s, T, sm).stab;
    double d = 0.0;
    for (int t = 0; t < nt.n_zf; ++t) d += (double)s_zfh[t] * (((s >> s_zf[t]) & 1ull) ? 1.0 : -1.0);
    for (int t = 0; t < nt.n_zz; ++t) {
      const int2 p = s_zz[t];
      d += (double)s_zzJ[t] * ((((s >> p.x) ^ (s >> p.y)) & 1ull) ? -1.0 : 1.0);
    }
    double acc = d * x[r];
    for (int k = 0; k < nt.n_moves; ++k) {
      const int2 p = s_ij[k];
      if (!(((s >> p.x) ^ (s >> p.y)) & 1ull)) continue;   // exchange of anti-parallel spins only
      const EdOrbit o = ed_orbit(s ^ s_mask[k], T, sm);
      if (!o.ok) continue;                                 // orbit outside the sector
      const int64_t q = ed_rep_index(o.m, T, sm, off, reps);
      if (q < 0) {
        ++miss;
        continue;
      }
      const double f = (double)s_c[k] * sqrt((double)o.stab * inv_stab);
      acc += (o.neg ? -f : f) * x[q];
    }
    y[r] = acc;
  }
  if (miss) atomicAdd(missing, miss);
}

namespace {
int ed_torus_setup(int lx, int ly, int n_up, int parity, int kx, int ky, EdTorus* T) {
  QES_ARG_CHECK(lx >= 1 && ly >= 1 && lx * ly <= 62, "qes_ed_symm: need 1 <= lx * ly <= 62");
  const int ns = lx * ly;
  QES_ARG_CHECK(n_up >= 0 && n_up <= ns && n_up < ED_BINOM_K, "qes_ed_symm: need 0 <= n_up <= min(ns, 32)");
  QES_ARG_CHECK(parity == 0 || ((parity == 1 || parity == -1) && 2 * n_up == ns),
                "qes_ed_symm: spin-flip parity needs ns = 2 n_up");
  QES_ARG_CHECK((kx == 0 || (kx == 1 && lx % 2 == 0)) && (ky == 0 || (ky == 1 && ly % 2 == 0)),
                "qes_ed_symm: momentum 0 (k = 0) or pi (k = 1) per axis; pi needs an even side");
  std::vector<uint64_t> C;
  ed_binomials(C);
  T->lx = lx;
  T->ly = ly;
  T->ns = ns;
  T->n_up = n_up;
  T->bits = parity ? ns - 1 : ns;
  T->parity = parity;
  T->kx = kx;
  T->ky = ky;
  T->full = (1ull << ns) - 1ull;
  T->n_ranks = C[(size_t)T->bits * ED_BINOM_K + n_up];
  if (T->n_ranks > ED_SYMM_MAX_RANKS) {
    qes_set_last_message("qes_ed_symm: more than 2^37 S^z states to enumerate");
    return QES_ERR_SIZE;
  }
  T->n_buckets = (T->n_ranks + 31) / 32;
  T->n_tiles = (T->n_buckets + ED_SCAN_TILE - 1) / ED_SCAN_TILE;
  return QES_OK;
}

size_t ed_al(size_t x) { return (x + 255) & ~(size_t)255; }

struct EdSymmLayout {
  size_t binom, part, miss, tsum, off, reps, v, vp, w, end;
};

// dim = 0: the dimension query (binomials and partial sums only)
EdSymmLayout ed_symm_layout(const EdTorus& T, uint64_t dim) {
  EdSymmLayout L{};
  size_t p = 0;
  L.binom = p;
  p += ed_al((size_t)ED_BINOM_N * ED_BINOM_K * sizeof(uint64_t));
  L.part = p;
  p += ed_al(ED_BLOCKS * sizeof(double));
  L.miss = p;
  p += 256;
  if (dim == 0) {
    L.end = p;
    return L;
  }
  L.tsum = p;
  p += ed_al((size_t)T.n_tiles * sizeof(unsigned long long));
  L.off = p;
  p += ed_al((size_t)(T.n_buckets + 1) * sizeof(uint32_t));
  L.reps = p;
  p += ed_al((size_t)dim * sizeof(uint64_t));
  L.v = p;
  p += ed_al((size_t)dim * sizeof(double));
  L.vp = p;
  p += ed_al((size_t)dim * sizeof(double));
  L.w = p;
  p += ed_al((size_t)dim * sizeof(double));
  L.end = p;
  return L;
}

int ed_sum_u64(const unsigned long long* dpart, cudaStream_t st, uint64_t* out) {
  std::vector<unsigned long long> h(ED_BLOCKS);
  QES_CUDA_CHECK(cudaMemcpyAsync(h.data(), dpart, ED_BLOCKS * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
  QES_CUDA_CHECK(cudaStreamSynchronize(st));
  uint64_t s = 0;
  for (int q = 0; q < ED_BLOCKS; ++q) s += h[q];
  *out = s;
  return QES_OK;
}

// Number of representatives (the sector dimension); one enumeration pass.
int ed_symm_count(const EdTorus& T, char* ws, uint32_t* cnt, cudaStream_t st, uint64_t* dim) {
  const EdSymmLayout L = ed_symm_layout(T, 0);
  std::vector<uint64_t> C;
  ed_binomials(C);
  uint64_t* binom = reinterpret_cast<uint64_t*>(ws + L.binom);
  QES_CUDA_CHECK(cudaMemcpyAsync(binom, C.data(), C.size() * sizeof(uint64_t), cudaMemcpyHostToDevice, st));
  auto* part = reinterpret_cast<unsigned long long*>(ws + L.part);
  ed_symm_count_kernel<<<ED_BLOCKS, ED_THREADS, 0, st>>>(T, binom, cnt, part);
  QES_LAUNCH_CHECK();
  return ed_sum_u64(part, st, dim);
}

// The Hamiltonian must conserve S^z with real elements (anti-parallel pair moves, real
// coefficients) and commute with the translations: its bonds and fields map onto themselves
// under T(1, 0) and T(0, 1).
int ed_symm_check_terms(const EdTorus& T, const qes_hamiltonian* ham, cudaStream_t st) {
  const int nm = ham->n_moves, nz = ham->n_zz, nf = ham->n_zfield;
  std::vector<int32_t> mi(nm), mj(nm), mk(nm), zi(nz), zj(nz), fs(nf);
  std::vector<float> mc((size_t)nm * 4), zJ(nz), fh(nf);
  if (nm > 0) {
    QES_ARG_CHECK(ham->move_i && ham->move_j && ham->move_kind && ham->move_coef, "qes_ed_symm: null move arrays");
    QES_CUDA_CHECK(cudaMemcpyAsync(mi.data(), ham->move_i, nm * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    QES_CUDA_CHECK(cudaMemcpyAsync(mj.data(), ham->move_j, nm * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    QES_CUDA_CHECK(cudaMemcpyAsync(mk.data(), ham->move_kind, nm * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    QES_CUDA_CHECK(cudaMemcpyAsync(mc.data(), ham->move_coef, mc.size() * sizeof(float), cudaMemcpyDeviceToHost, st));
  }
  if (nz > 0) {
    QES_ARG_CHECK(ham->zz_i && ham->zz_j && ham->zz_J, "qes_ed_symm: null zz arrays");
    QES_CUDA_CHECK(cudaMemcpyAsync(zi.data(), ham->zz_i, nz * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    QES_CUDA_CHECK(cudaMemcpyAsync(zj.data(), ham->zz_j, nz * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    QES_CUDA_CHECK(cudaMemcpyAsync(zJ.data(), ham->zz_J, nz * sizeof(float), cudaMemcpyDeviceToHost, st));
  }
  if (nf > 0) {
    QES_ARG_CHECK(ham->zf_site && ham->zf_h, "qes_ed_symm: null field arrays");
    QES_CUDA_CHECK(cudaMemcpyAsync(fs.data(), ham->zf_site, nf * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    QES_CUDA_CHECK(cudaMemcpyAsync(fh.data(), ham->zf_h, nf * sizeof(float), cudaMemcpyDeviceToHost, st));
  }
  QES_CUDA_CHECK(cudaStreamSynchronize(st));
  auto site_ok = [&](int i) { return i >= 0 && i < T.ns; };
  std::map<std::pair<int, int>, double> mv, zz;
  std::map<int, double> zf;
  for (int k = 0; k < nm; ++k) {
    QES_ARG_CHECK(mk[k] == QES_MOVE_PAIR_ANTI, "qes_ed_symm: the Hamiltonian does not conserve S^z");
    QES_ARG_CHECK(mc[4 * k + 1] == 0.f && mc[4 * k + 2] == 0.f && mc[4 * k + 3] == 0.f,
                  "qes_ed_symm: complex matrix elements");
    QES_ARG_CHECK(site_ok(mi[k]) && site_ok(mj[k]) && mi[k] != mj[k], "qes_ed_symm: bad move sites");
    mv[{std::min(mi[k], mj[k]), std::max(mi[k], mj[k])}] += mc[4 * k];
  }
  for (int t = 0; t < nz; ++t) {
    QES_ARG_CHECK(site_ok(zi[t]) && site_ok(zj[t]), "qes_ed_symm: bad zz sites");
    zz[{std::min(zi[t], zj[t]), std::max(zi[t], zj[t])}] += zJ[t];
  }
  for (int t = 0; t < nf; ++t) {
    QES_ARG_CHECK(site_ok(fs[t]), "qes_ed_symm: bad field site");
    zf[fs[t]] += fh[t];
  }
  auto same = [](double a, double b) { return fabs(a - b) <= 1e-6 * std::max(1.0, std::max(fabs(a), fabs(b))); };
  const int gens[2][2] = {{1, 0}, {0, 1}};
  for (const auto& g : gens) {
    auto tr = [&](int i) { return (i % T.lx + g[0]) % T.lx + T.lx * ((i / T.lx + g[1]) % T.ly); };
    for (const auto* m : {&mv, &zz}) {
      for (const auto& e : *m) {
        const int a = tr(e.first.first), b = tr(e.first.second);
        const auto it = m->find({std::min(a, b), std::max(a, b)});
        QES_ARG_CHECK(it != m->end() && same(it->second, e.second),
                      "qes_ed_symm: the Hamiltonian is not translation invariant");
      }
    }
    for (const auto& e : zf) {
      const auto it = zf.find(tr(e.first));
      QES_ARG_CHECK(it != zf.end() && same(it->second, e.second),
                    "qes_ed_symm: the Hamiltonian is not translation invariant");
    }
  }
  return QES_OK;
}
}  // namespace

extern "C" int qes_ed_symm_workspace_bytes(int lx, int ly, int n_up, int parity, int kx, int ky, uint64_t dim,
                                           size_t* bytes) {
  QES_ARG_CHECK(bytes, "qes_ed_symm_workspace_bytes: null output");
  EdTorus T{};
  int rc = ed_torus_setup(lx, ly, n_up, parity, kx, ky, &T);
  if (rc) return rc;
  *bytes = ed_symm_layout(T, dim).end;
  return QES_OK;
}

extern "C" int qes_ed_symm_dim(int lx, int ly, int n_up, int parity, int kx, int ky, uint64_t* dim, void* workspace,
                               size_t workspace_bytes, void* stream) {
  QES_ARG_CHECK(dim, "qes_ed_symm_dim: null output");
  EdTorus T{};
  int rc = ed_torus_setup(lx, ly, n_up, parity, kx, ky, &T);
  if (rc) return rc;
  if (!workspace || workspace_bytes < ed_symm_layout(T, 0).end) {
    qes_set_last_message("qes_ed_symm_dim: workspace too small");
    return QES_ERR_WORKSPACE;
  }
  return ed_symm_count(T, (char*)workspace, nullptr, (cudaStream_t)stream, dim);
}

extern "C" int qes_ed_lanczos_symm(int lx, int ly, int n_up, int parity, int kx, int ky, const qes_hamiltonian* ham,
                                   int max_iter, double tol, uint64_t seed, double* e0_out, int* iterations_out,
                                   uint64_t* dim_out, void* workspace, size_t workspace_bytes, void* stream) {
  QES_ARG_CHECK(ham && e0_out && max_iter >= 2 && tol > 0.0, "qes_ed_lanczos_symm: bad args");
  QES_ARG_CHECK(ham->n_moves >= 0 && ham->n_moves <= ED_MAX_TERMS && ham->n_zz >= 0 && ham->n_zz <= ED_MAX_TERMS &&
                    ham->n_zfield >= 0 && ham->n_zfield <= ED_MAX_TERMS,
                "qes_ed_lanczos_symm: too many terms");
  QES_ARG_CHECK(!(parity != 0 && ham->n_zfield > 0), "qes_ed_lanczos_symm: a z field breaks the spin-flip parity");
  EdTorus T{};
  int rc = ed_torus_setup(lx, ly, n_up, parity, kx, ky, &T);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  if ((rc = ed_symm_check_terms(T, ham, st))) return rc;
  const EdSymmLayout L1 = ed_symm_layout(T, 1);
  if (!workspace || workspace_bytes < L1.off + (size_t)(T.n_buckets + 1) * sizeof(uint32_t)) {
    qes_set_last_message("qes_ed_lanczos_symm: workspace too small");
    return QES_ERR_WORKSPACE;
  }
  char* ws = (char*)workspace;
  uint32_t* off = reinterpret_cast<uint32_t*>(ws + L1.off);
  uint64_t dim = 0;
  if ((rc = ed_symm_count(T, ws, off, st, &dim))) return rc;
  QES_ARG_CHECK(dim >= 1, "qes_ed_lanczos_symm: empty sector");
  if (dim >= (1ull << 32)) {
    qes_set_last_message("qes_ed_lanczos_symm: more than 2^32 representatives");
    return QES_ERR_SIZE;
  }
  const EdSymmLayout L = ed_symm_layout(T, dim);
  if (workspace_bytes < L.end) {
    qes_set_last_message("qes_ed_lanczos_symm: workspace too small for the sector (qes_ed_symm_dim, then "
                         "qes_ed_symm_workspace_bytes with that dimension)");
    return QES_ERR_WORKSPACE;
  }
  const uint64_t* binom = reinterpret_cast<const uint64_t*>(ws + L.binom);
  auto* tsum = reinterpret_cast<unsigned long long*>(ws + L.tsum);
  auto* miss = reinterpret_cast<unsigned long long*>(ws + L.miss);
  auto* reps = reinterpret_cast<uint64_t*>(ws + L.reps);
  const int tgrid = (int)std::min<uint64_t>(T.n_tiles, ED_BLOCKS);
  ed_tile_sum_kernel<<<tgrid, ED_THREADS, 0, st>>>(T.n_buckets, T.n_tiles, off, tsum);
  QES_LAUNCH_CHECK();
  std::vector<unsigned long long> toff(T.n_tiles);
  QES_CUDA_CHECK(cudaMemcpyAsync(toff.data(), tsum, T.n_tiles * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
  QES_CUDA_CHECK(cudaStreamSynchronize(st));
  unsigned long long run = 0;
  for (auto& t : toff) {
    const unsigned long long c = t;
    t = run;
    run += c;
  }
  QES_ARG_CHECK(run == dim, "qes_ed_lanczos_symm: inconsistent representative count");
  QES_CUDA_CHECK(cudaMemcpyAsync(tsum, toff.data(), T.n_tiles * sizeof(unsigned long long), cudaMemcpyHostToDevice, st));
  ed_tile_scan_kernel<<<tgrid, ED_THREADS, 0, st>>>(T.n_buckets, T.n_tiles, off, tsum, dim);
  ed_symm_fill_kernel<<<ED_BLOCKS, ED_THREADS, 0, st>>>(T, binom, off, reps);
  QES_LAUNCH_CHECK_N(2);
  QES_CUDA_CHECK(cudaMemsetAsync(miss, 0, sizeof(unsigned long long), st));
  double* v = reinterpret_cast<double*>(ws + L.v);
  double* vp = reinterpret_cast<double*>(ws + L.vp);
  double* w = reinterpret_cast<double*>(ws + L.w);
  double* part = reinterpret_cast<double*>(ws + L.part);
  const EdTerms nt{ham->n_moves, ham->n_zz, ham->n_zfield};
  auto matvec = [&](const double* x, double* y) {
    ed_symm_matvec_kernel<<<ED_BLOCKS, ED_THREADS, 0, st>>>(T, dim, nt, ham->move_i, ham->move_j,
                                                            (const float4*)ham->move_coef, ham->zf_site, ham->zf_h,
                                                            ham->zz_i, ham->zz_j, ham->zz_J, binom, off, reps, x, y,
                                                            miss);
  };
  rc = ed_lanczos_loop(dim, matvec, v, vp, w, part, max_iter, tol, seed, st, e0_out, iterations_out);
  unsigned long long h_miss = 0;
  QES_CUDA_CHECK(cudaMemcpyAsync(&h_miss, miss, sizeof(h_miss), cudaMemcpyDeviceToHost, st));
  QES_CUDA_CHECK(cudaStreamSynchronize(st));
  if (dim_out) *dim_out = dim;
  QES_ARG_CHECK(h_miss == 0, "qes_ed_lanczos_symm: a connected representative is missing from the list");
  return rc;
}
