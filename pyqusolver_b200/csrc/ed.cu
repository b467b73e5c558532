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
    ed_launch_matvec(ns, ham, v, w, st);
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
  std::vector<double> hpart(ED_BLOCKS), alpha, beta;
  ed_init_kernel<<<ED_BLOCKS, ED_THREADS, 0, st>>>(dim, (uint32_t)seed, (uint32_t)(seed >> 32), v, vp, part);
  QES_LAUNCH_CHECK();
  double nrm2 = 0.0;
  if ((rc = ed_sum(part, hpart.data(), st, &nrm2))) return rc;
  ed_scale_kernel<<<ED_BLOCKS, ED_THREADS, 0, st>>>(dim, 1.0 / sqrt(nrm2), v);
  QES_LAUNCH_CHECK();
  const EdTerms nt{ham->n_moves, ham->n_zz, ham->n_zfield};
  double e_prev = 0.0, e = 0.0, b_prev = 0.0;
  int it = 0;
  bool conv = false;
  for (; it < max_iter; ++it) {
    ed_sector_matvec_kernel<<<ED_BLOCKS, ED_THREADS, 0, st>>>(sec, dim, nt, ham->move_i, ham->move_j,
                                                              (const float4*)ham->move_coef, ham->zf_site, ham->zf_h,
                                                              ham->zz_i, ham->zz_j, ham->zz_J, binom, v, w);
    ed_dot_kernel<<<ED_BLOCKS, ED_THREADS, 0, st>>>(dim, v, w, part);
    QES_LAUNCH_CHECK_N(2);
    double a = 0.0;
    if ((rc = ed_sum(part, hpart.data(), st, &a))) return rc;
    alpha.push_back(a);
    ed_axpy_norm_kernel<<<ED_BLOCKS, ED_THREADS, 0, st>>>(dim, a, b_prev, v, vp, w, part);
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
    ed_shift_kernel<<<ED_BLOCKS, ED_THREADS, 0, st>>>(dim, 1.0 / b, vp, v, w);
    QES_LAUNCH_CHECK();
    b_prev = b;
  }
  *e0_out = e;
  if (iterations_out) *iterations_out = it;
  return conv ? QES_OK : QES_ERR_NOT_CONVERGED;
}
