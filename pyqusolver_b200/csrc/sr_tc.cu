// Tensor-core (tcgen05) halves of the structured SR matvec.
//
//   ov :  Z = Sigma V          (128 samples x Kp sites) . (Kp sites x Np)  -> TMEM
//         w_s = sum_m t_sm (vb_m + Z_sm) + sigma_s . va          (epilogue, CUDA cores)
//   ohu:  G_W = Sigma^T Q      (128 sites x KC samples) . (KC samples x Np) -> TMEM
//         Q_sm = conj(t_sm) u_s, u_s = (w_s - mean w) / Ns      (staged by CUDA cores)
//
// Sigma (+-1) is exact in BF16.  The other operand is split x = hi + lo into
// two BF16 terms accumulated into the same FP32 TMEM accumulator, which keeps
// ~16 significant bits of the float32 value (the product with +-1 adds no
// rounding).  Complex operands are laid out as Np = 2*Mp rows: real parts in
// rows [0, Mp), imaginary parts in [Mp, 2Mp); the two halves are two MMAs of
// N = Mp into TMEM columns [0, Mp) and [im_off, im_off + Mp).
//
// Every wait on an mbarrier is bounded; on time-out the kernel records an
// error code in *status, still waits (bounded) for what it issued, frees its
// TMEM and returns.  The host reads *status after the solve.
#include "common.cuh"
#include "sr_tc.h"
#include "umma.cuh"

#include <cuda_bf16.h>

namespace {

constexpr uint32_t kWaitLimit = 1u << 22;     // try_wait polls before giving up
constexpr int kThreads = 128;                  // 4 warps <-> 4 TMEM lane quarters

__device__ __forceinline__ uint16_t bf16_bits(float x) {
  return __bfloat16_as_ushort(__float2bfloat16_rn(x));
}
__device__ __forceinline__ float bf16_val(uint16_t b) { return __bfloat162float(__ushort_as_bfloat16(b)); }
__device__ __forceinline__ void split_bf16(float x, uint16_t& hi, uint16_t& lo) {
  hi = bf16_bits(x);
  lo = bf16_bits(x - bf16_val(hi));
}

__device__ __forceinline__ uint32_t pack2(uint16_t a, uint16_t b) { return (uint32_t)a | ((uint32_t)b << 16); }

__device__ __forceinline__ void record_error(int* status, int code) {
  if (status) atomicCAS(status, 0, code);
}

// values of V (float64 / complex128) as float
__device__ __forceinline__ float vre(const double* v, int64_t k) { return (float)v[k]; }
__device__ __forceinline__ float vre(const double2* v, int64_t k) { return (float)v[k].x; }
__device__ __forceinline__ float vim(const double*, int64_t) { return 0.f; }
__device__ __forceinline__ float vim(const double2* v, int64_t k) { return (float)v[k].y; }

}  // namespace

// ------------------------------------------------------------------------------------------------
// per-step operands: Sigma in rows-of-samples tiles and in rows-of-sites chunks
// ------------------------------------------------------------------------------------------------
// sig_rows: tile t holds samples [128t, 128t+128) x Kp sites; sig_cols: chunk c holds 128 sites x
// samples [KC c, KC c + KC).  Padding (sites >= ns, samples >= Ns) is zero.
__global__ void tc_sigma_rows_kernel(int ns, int Kp, int64_t n_samples, int n_tiles, const uint32_t* __restrict__ bits,
                                     uint16_t* __restrict__ out) {
  const int nw = n_words(ns);
  const int64_t items = (int64_t)n_tiles * 128 * (Kp / 8);
  for (int64_t it = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; it < items; it += (int64_t)gridDim.x * blockDim.x) {
    const int k8 = (int)(it % (Kp / 8));
    const int r = (int)((it / (Kp / 8)) % 128);
    const int64_t t = it / ((int64_t)(Kp / 8) * 128);
    const int64_t s = t * 128 + r;
    uint16_t v[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int i = 8 * k8 + q;
      v[q] = 0;
      if (s < n_samples && i < ns) v[q] = ((bits[s * nw + (i >> 5)] >> (i & 31)) & 1u) ? 0x3F80u : 0xBF80u;
    }
    uint4 pk = make_uint4(pack2(v[0], v[1]), pack2(v[2], v[3]), pack2(v[4], v[5]), pack2(v[6], v[7]));
    uint8_t* base = reinterpret_cast<uint8_t*>(out) + (size_t)t * 128 * Kp * 2;
    *reinterpret_cast<uint4*>(base + umma::kmajor_offset(r, 8 * k8, 128)) = pk;
  }
}

__global__ void tc_sigma_cols_kernel(int ns, int KC, int64_t n_samples, int n_chunks, const uint32_t* __restrict__ bits,
                                     uint16_t* __restrict__ out) {
  const int nw = n_words(ns);
  const int64_t items = (int64_t)n_chunks * 128 * (KC / 8);
  for (int64_t it = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; it < items; it += (int64_t)gridDim.x * blockDim.x) {
    const int k8 = (int)(it % (KC / 8));
    const int r = (int)((it / (KC / 8)) % 128);          // site
    const int64_t c = it / ((int64_t)(KC / 8) * 128);
    uint16_t v[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int64_t s = c * KC + 8 * k8 + q;
      v[q] = 0;
      if (s < n_samples && r < ns) v[q] = ((bits[s * nw + (r >> 5)] >> (r & 31)) & 1u) ? 0x3F80u : 0xBF80u;
    }
    uint4 pk = make_uint4(pack2(v[0], v[1]), pack2(v[2], v[3]), pack2(v[4], v[5]), pack2(v[6], v[7]));
    uint8_t* base = reinterpret_cast<uint8_t*>(out) + (size_t)c * 128 * KC * 2;
    *reinterpret_cast<uint4*>(base + umma::kmajor_offset(r, 8 * k8, 128)) = pk;
  }
}

// ------------------------------------------------------------------------------------------------
// per-iteration B operand of ov: rows n (hidden, re then im) x Kp sites, hi and lo terms
// ------------------------------------------------------------------------------------------------
template <class V>
__global__ void tc_build_v_kernel(int ns, int nh, int Kp, int Mp, int Np, bool cplx, const V* __restrict__ v,
                                  uint16_t* __restrict__ bhi, uint16_t* __restrict__ blo) {
  const int items = Np * (Kp / 8);
  const V* vW = v + ns + nh;
  for (int it = blockIdx.x * blockDim.x + threadIdx.x; it < items; it += gridDim.x * blockDim.x) {
    const int k8 = it % (Kp / 8);
    const int n = it / (Kp / 8);
    const bool im = cplx && n >= Mp;
    const int m = im ? n - Mp : n;
    uint16_t h[8], l[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int i = 8 * k8 + q;
      float x = 0.f;
      if (i < ns && m < nh) {
        const int64_t k = (int64_t)i * nh + m;
        x = im ? vim(vW, k) : vre(vW, k);
      }
      split_bf16(x, h[q], l[q]);
    }
    const uint32_t off = umma::kmajor_offset(n, 8 * k8, Np);
    *reinterpret_cast<uint4*>(reinterpret_cast<uint8_t*>(bhi) + off) =
        make_uint4(pack2(h[0], h[1]), pack2(h[2], h[3]), pack2(h[4], h[5]), pack2(h[6], h[7]));
    *reinterpret_cast<uint4*>(reinterpret_cast<uint8_t*>(blo) + off) =
        make_uint4(pack2(l[0], l[1]), pack2(l[2], l[3]), pack2(l[4], l[5]), pack2(l[6], l[7]));
  }
}

// ------------------------------------------------------------------------------------------------
// ov: one CTA per 128-sample tile
// ------------------------------------------------------------------------------------------------
template <class T, class V>
__global__ void __launch_bounds__(kThreads) tc_ov_kernel(TcDims d, int64_t n_samples, const uint32_t* __restrict__ bits,
                                                         const T* __restrict__ tanh_theta, const V* __restrict__ v,
                                                         const uint16_t* __restrict__ sig_rows,
                                                         const uint16_t* __restrict__ bhi,
                                                         const uint16_t* __restrict__ blo, float2* __restrict__ w_out,
                                                         double2* __restrict__ wsum_part, int* __restrict__ status) {
  extern __shared__ __align__(128) uint8_t smem[];
  constexpr bool CPLX = ScalarTraits<T>::is_complex;
  const int ns = d.ns, nh = d.nh, Kp = d.Kp, Mp = d.Mp, Np = d.Np;
  const uint32_t a_bytes = 128u * Kp * 2u, b_bytes = (uint32_t)Np * Kp * 2u;
  uint8_t* sA = smem;
  uint8_t* sBh = sA + a_bytes;
  uint8_t* sBl = sBh + b_bytes;
  T* s_vb = reinterpret_cast<T*>(sBl + b_bytes);                         // nh
  T* s_va = s_vb + nh;                                                    // ns
  uint64_t* bars = reinterpret_cast<uint64_t*>(reinterpret_cast<uint8_t*>(s_va + ns) +
                                               ((16 - (reinterpret_cast<uintptr_t>(s_va + ns) & 15)) & 15));
  uint32_t* tslot = reinterpret_cast<uint32_t*>(bars + 2);
  __shared__ double2 red[kThreads / 32];
  __shared__ int s_issued;

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int tile = blockIdx.x;
  if (tid == 0) {
    umma::mbar_init(&bars[0], 1);
    umma::mbar_init(&bars[1], 1);
    umma::fence_mbar_init();
  }
  if (warp == 0) {
    umma::tmem_alloc(tslot, d.tmem_cols);
    umma::tmem_relinquish();
  }
  // small vectors of the direction (float)
  for (int m = tid; m < nh; m += kThreads) {
    if constexpr (CPLX) s_vb[m] = make_float2(vre(v, ns + m), vim(v, ns + m));
    else s_vb[m] = vre(v, ns + m);
  }
  for (int i = tid; i < ns; i += kThreads) {
    if constexpr (CPLX) s_va[i] = make_float2(vre(v, i), vim(v, i));
    else s_va[i] = vre(v, i);
  }
  umma::tc_fence_before();
  __syncthreads();
  umma::tc_fence_after();
  const uint32_t tbase = *tslot;
  bool ok = true;
  if (tid == 0) {
    umma::mbar_arrive_expect_tx(&bars[0], a_bytes + 2 * b_bytes);
    umma::bulk_g2s(sA, reinterpret_cast<const uint8_t*>(sig_rows) + (size_t)tile * a_bytes, a_bytes, &bars[0]);
    umma::bulk_g2s(sBh, bhi, b_bytes, &bars[0]);
    umma::bulk_g2s(sBl, blo, b_bytes, &bars[0]);
    if (!umma::mbar_wait(&bars[0], 0, kWaitLimit)) {
      ok = false;
      record_error(status, QES_ERR_TIMEOUT);
    }
    if (ok) {
      umma::tc_fence_after();
      const uint32_t idesc = umma::idesc_bf16_f32(128, Mp);
      const uint32_t aaddr = umma::smem_u32(sA), bh = umma::smem_u32(sBh), bl = umma::smem_u32(sBl);
      const int halves = CPLX ? 2 : 1;
      for (int j = 0; j < Kp / 16; ++j) {
        const uint64_t ad = umma::smem_desc(aaddr + 2u * j * 128u * 16u, 128u * 16u, 128u);
        for (int term = 0; term < 2; ++term) {
          const uint32_t bb = term ? bl : bh;
          for (int h = 0; h < halves; ++h) {
            const uint64_t bd = umma::smem_desc(bb + (uint32_t)h * (Mp / 8) * 128u + 2u * j * Np * 16u, Np * 16u, 128u);
            umma::mma_bf16(tbase + (uint32_t)h * d.im_off, ad, bd, idesc, (j > 0 || term > 0) ? 1u : 0u);
          }
        }
      }
      umma::mma_commit(&bars[1]);
    } else {
      umma::mbar_wait(&bars[0], 0, kWaitLimit);      // let the copies in flight land before exit
    }
    s_issued = ok ? 1 : 0;
  }
  __syncthreads();
  // every thread waits (bounded) for this CTA's own MMAs, when they were issued
  if (s_issued && !umma::mbar_wait(&bars[1], 0, kWaitLimit)) record_error(status, QES_ERR_TIMEOUT);
  umma::tc_fence_after();

  // epilogue: this thread owns sample row 32*warp + lane of the tile
  const int row = 32 * warp + lane;
  const int64_t s = (int64_t)tile * 128 + row;
  const bool sval = s < n_samples;
  const int64_t sc = sval ? s : 0;
  T acc = ScalarTraits<T>::zero();
  const T* trow = tanh_theta + sc * nh;
  const uint32_t lane_addr = tbase + ((uint32_t)(32 * warp) << 16);
  for (int c0 = 0; c0 < Mp; c0 += 16) {
    float zr[16], zi[16];
    umma::tmem_ld16(lane_addr + c0, zr);
    if constexpr (CPLX) umma::tmem_ld16(lane_addr + d.im_off + c0, zi);
#pragma unroll
    for (int q = 0; q < 16; ++q) {
      const int m = c0 + q;
      if (m < nh) {
        if constexpr (CPLX) {
          const float2 z = make_float2(zr[q] + s_vb[m].x, zi[q] + s_vb[m].y);
          acc = addx(acc, mulx(trow[m], z));
        } else {
          acc += trow[m] * (zr[q] + s_vb[m]);
        }
      }
    }
  }
  const uint32_t* wrd = bits + sc * n_words(ns);
  for (int i = 0; i < ns; ++i) {
    const float sg = ((wrd[i >> 5] >> (i & 31)) & 1u) ? 1.f : -1.f;
    acc = addx(acc, scal(sg, s_va[i]));
  }
  float2 wv = sval ? to_c(acc) : make_float2(0.f, 0.f);
  if (sval) w_out[s] = wv;
  double2 ps = make_double2(wv.x, wv.y);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    ps.x += __shfl_xor_sync(0xffffffffu, ps.x, o);
    ps.y += __shfl_xor_sync(0xffffffffu, ps.y, o);
  }
  if (lane == 0) red[warp] = ps;
  umma::tc_fence_before();
  __syncthreads();
  if (tid == 0) {
    double2 t = make_double2(0.0, 0.0);
    for (int q = 0; q < kThreads / 32; ++q) { t.x += red[q].x; t.y += red[q].y; }
    wsum_part[tile] = t;
  }
  if (warp == 0) umma::tmem_dealloc(tbase, d.tmem_cols);
}

// ------------------------------------------------------------------------------------------------
// ohu: one CTA per KC-sample chunk; writes one P-vector of partial sums
// ------------------------------------------------------------------------------------------------
template <class T>
__global__ void __launch_bounds__(kThreads) tc_ohu_kernel(TcDims d, int64_t n_samples, const uint32_t* __restrict__ bits,
                                                          const T* __restrict__ tanh_theta, const float2* __restrict__ w,
                                                          const double2* __restrict__ wsum_part, int wsum_n, double scale,
                                                          const uint16_t* __restrict__ sig_cols, T* __restrict__ partial,
                                                          int* __restrict__ status) {
  extern __shared__ __align__(128) uint8_t smem[];
  constexpr bool CPLX = ScalarTraits<T>::is_complex;
  const int ns = d.ns, nh = d.nh, Mp = d.Mp, Np = d.Np, KC = d.KC;
  const uint32_t a_bytes = 128u * KC * 2u, b_bytes = (uint32_t)Np * KC * 2u;
  uint8_t* sA = smem;
  uint8_t* sBh = sA + a_bytes;
  uint8_t* sBl = sBh + b_bytes;
  T* s_u = reinterpret_cast<T*>(sBl + b_bytes);            // KC
  T* s_gb = s_u + KC;                                      // nh (partial g_b of this chunk)
  uint64_t* bars = reinterpret_cast<uint64_t*>(reinterpret_cast<uint8_t*>(s_gb + nh) +
                                               ((16 - (reinterpret_cast<uintptr_t>(s_gb + nh) & 15)) & 15));
  uint32_t* tslot = reinterpret_cast<uint32_t*>(bars + 2);
  __shared__ double2 s_mean;
  __shared__ int s_issued;

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int chunk = blockIdx.x;
  const int64_t s0 = (int64_t)chunk * KC;
  const int64_t P = (int64_t)ns + nh + (int64_t)ns * nh;
  if (tid == 0) {
    umma::mbar_init(&bars[0], 1);
    umma::mbar_init(&bars[1], 1);
    umma::fence_mbar_init();
    double2 t = make_double2(0.0, 0.0);
    if (wsum_part && wsum_n > 0) {
      for (int q = 0; q < wsum_n; ++q) { t.x += wsum_part[q].x; t.y += wsum_part[q].y; }
      t.x /= (double)n_samples;
      t.y /= (double)n_samples;
    } else if (wsum_part) {
      t = wsum_part[0];              // the mean itself
    }
    s_mean = t;
  }
  if (warp == 0) {
    umma::tmem_alloc(tslot, d.tmem_cols);
    umma::tmem_relinquish();
  }
  umma::tc_fence_before();
  __syncthreads();
  umma::tc_fence_after();
  const uint32_t tbase = *tslot;
  if (tid == 0) {
    umma::mbar_arrive_expect_tx(&bars[0], a_bytes);
    umma::bulk_g2s(sA, reinterpret_cast<const uint8_t*>(sig_cols) + (size_t)chunk * a_bytes, a_bytes, &bars[0]);
  }
  // u_s = (w_s - mean) * scale, zero beyond Ns
  const float mr = (float)s_mean.x, mi = (float)s_mean.y, fs = (float)scale;
  for (int k = tid; k < KC; k += kThreads) {
    const int64_t s = s0 + k;
    T u = ScalarTraits<T>::zero();
    if (s < n_samples) {
      const float2 wv = w[s];
      if constexpr (CPLX) u = make_float2((wv.x - mr) * fs, (wv.y - mi) * fs);
      else u = (wv.x - mr) * fs;
    }
    s_u[k] = u;
  }
  for (int m = tid; m < nh; m += kThreads) s_gb[m] = ScalarTraits<T>::zero();
  __syncthreads();
  // Q = conj(t) u, split into hi/lo, written as B rows (re: m, im: Mp + m) x KC samples;
  // item (m, k8) covers 8 consecutive samples -> one 16-byte store per row and term
  const int items = Mp * (KC / 8);
  for (int it = tid; it < items; it += kThreads) {
    const int m = it % Mp, k8 = it / Mp;
    uint16_t rh[8], rl[8], ih[8], il[8];
    T qs = ScalarTraits<T>::zero();
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int k = 8 * k8 + q;
      const int64_t s = s0 + k;
      T qv = ScalarTraits<T>::zero();
      if (m < nh && s < n_samples) qv = mulx(conjx(tanh_theta[s * nh + m]), s_u[k]);
      qs = addx(qs, qv);
      const float qr = to_re(qv);
      split_bf16(qr, rh[q], rl[q]);
      if constexpr (CPLX) split_bf16(qv.y, ih[q], il[q]);
    }
    const uint32_t off = umma::kmajor_offset(m, 8 * k8, Np);
    *reinterpret_cast<uint4*>(sBh + off) = make_uint4(pack2(rh[0], rh[1]), pack2(rh[2], rh[3]), pack2(rh[4], rh[5]), pack2(rh[6], rh[7]));
    *reinterpret_cast<uint4*>(sBl + off) = make_uint4(pack2(rl[0], rl[1]), pack2(rl[2], rl[3]), pack2(rl[4], rl[5]), pack2(rl[6], rl[7]));
    if constexpr (CPLX) {
      const uint32_t offi = umma::kmajor_offset(Mp + m, 8 * k8, Np);
      *reinterpret_cast<uint4*>(sBh + offi) = make_uint4(pack2(ih[0], ih[1]), pack2(ih[2], ih[3]), pack2(ih[4], ih[5]), pack2(ih[6], ih[7]));
      *reinterpret_cast<uint4*>(sBl + offi) = make_uint4(pack2(il[0], il[1]), pack2(il[2], il[3]), pack2(il[4], il[5]), pack2(il[6], il[7]));
    }
    if (m < nh) {
      if constexpr (CPLX) {
        atomicAdd(&s_gb[m].x, qs.x);
        atomicAdd(&s_gb[m].y, qs.y);
      } else {
        atomicAdd(&s_gb[m], qs);
      }
    }
  }
  umma::fence_proxy_async_smem();     // generic-proxy stores -> visible to the tensor core
  __syncthreads();
  bool ok = true;
  if (tid == 0) {
    if (!umma::mbar_wait(&bars[0], 0, kWaitLimit)) {
      ok = false;
      record_error(status, QES_ERR_TIMEOUT);
    }
    if (ok) {
      umma::tc_fence_after();
      const uint32_t idesc = umma::idesc_bf16_f32(128, Mp);
      const uint32_t aaddr = umma::smem_u32(sA), bh = umma::smem_u32(sBh), bl = umma::smem_u32(sBl);
      const int halves = CPLX ? 2 : 1;
      for (int j = 0; j < KC / 16; ++j) {
        const uint64_t ad = umma::smem_desc(aaddr + 2u * j * 128u * 16u, 128u * 16u, 128u);
        for (int term = 0; term < 2; ++term) {
          const uint32_t bb = term ? bl : bh;
          for (int h = 0; h < halves; ++h) {
            const uint64_t bd = umma::smem_desc(bb + (uint32_t)h * (Mp / 8) * 128u + 2u * j * Np * 16u, Np * 16u, 128u);
            umma::mma_bf16(tbase + (uint32_t)h * d.im_off, ad, bd, idesc, (j > 0 || term > 0) ? 1u : 0u);
          }
        }
      }
      umma::mma_commit(&bars[1]);
    } else {
      umma::mbar_wait(&bars[0], 0, kWaitLimit);      // let the copy in flight land before exit
    }
    s_issued = ok ? 1 : 0;
  }
  // while the tensor core runs: g_a[i] = sum_s sigma_si u_s and g_b of this chunk
  T* out = partial + (int64_t)chunk * P;
  for (int i = tid; i < ns; i += kThreads) {
    T ga = ScalarTraits<T>::zero();
    for (int k = 0; k < KC; ++k) {
      const int64_t s = s0 + k;
      if (s >= n_samples) break;
      const float sg = ((bits[s * n_words(ns) + (i >> 5)] >> (i & 31)) & 1u) ? 1.f : -1.f;
      ga = addx(ga, scal(sg, s_u[k]));
    }
    out[i] = ga;
  }
  for (int m = tid; m < nh; m += kThreads) out[ns + m] = s_gb[m];
  __syncthreads();
  if (s_issued && !umma::mbar_wait(&bars[1], 0, kWaitLimit)) record_error(status, QES_ERR_TIMEOUT);
  umma::tc_fence_after();
  const int i = 32 * warp + lane;                         // site row of the accumulator
  const uint32_t lane_addr = tbase + ((uint32_t)(32 * warp) << 16);
  for (int c0 = 0; c0 < Mp; c0 += 16) {
    float gr[16], gi[16];
    umma::tmem_ld16(lane_addr + c0, gr);
    if constexpr (CPLX) umma::tmem_ld16(lane_addr + d.im_off + c0, gi);
    if (i < ns) {
      T* row = out + ns + nh + (int64_t)i * nh;
#pragma unroll
      for (int q = 0; q < 16; ++q) {
        const int m = c0 + q;
        if (m < nh) {
          if constexpr (CPLX) row[m] = make_float2(gr[q], gi[q]);
          else row[m] = gr[q];
        }
      }
    }
  }
  umma::tc_fence_before();
  __syncthreads();
  if (warp == 0) umma::tmem_dealloc(tbase, d.tmem_cols);
}

// ------------------------------------------------------------------------------------------------
// host side
// ------------------------------------------------------------------------------------------------
static int pow2_at_least(int x) {
  int p = 32;
  while (p < x) p <<= 1;
  return p;
}

bool tc_plan(int dtype, int ns, int nh, int64_t n_samples, TcDims* d) {
  const bool cplx = dtype == QES_DTYPE_C64;
  TcDims t{};
  t.ns = ns;
  t.nh = nh;
  t.Kp = (ns + 15) / 16 * 16;
  t.Mp = (nh + 15) / 16 * 16;
  t.Np = cplx ? 2 * t.Mp : t.Mp;
  if (ns > 128 || t.Mp > 256 || n_samples < 1) return false;
  t.im_off = pow2_at_least(t.Mp);
  t.tmem_cols = cplx ? 2 * t.im_off : t.im_off;
  if (t.tmem_cols > 512) return false;
  const size_t tsz = cplx ? 8 : 4;
  const size_t ov_smem = 128u * t.Kp * 2 + 2u * t.Np * t.Kp * 2 + (ns + nh) * tsz + 64;
  if (ov_smem > kTcSmemLimit) return false;
  // largest multiple of 16 (<= 256) whose ohu shared memory fits
  int kc = 256;
  while (kc >= 16) {
    const size_t sm = 128u * kc * 2 + 2u * t.Np * kc * 2 + (kc + nh) * tsz + 64;
    if (sm <= kTcSmemLimit) break;
    kc -= 16;
  }
  if (kc < 16) return false;
  t.KC = kc;
  t.n_tiles = (int)((n_samples + 127) / 128);
  t.n_chunks = (int)((n_samples + kc - 1) / kc);
  t.ov_smem = (int)ov_smem;
  t.ohu_smem = (int)(128u * kc * 2 + 2u * t.Np * kc * 2 + (kc + nh) * tsz + 64);
  *d = t;
  return true;
}

size_t tc_workspace_bytes(const TcDims& d) {
  auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
  return al((size_t)d.n_tiles * 128 * d.Kp * 2) + al((size_t)d.n_chunks * 128 * d.KC * 2) +
         2 * al((size_t)d.Np * d.Kp * 2) + al((size_t)d.n_tiles * sizeof(double2)) + al(sizeof(int) * 4);
}

TcWork tc_layout(const TcDims& d, char* base) {
  auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
  TcWork w{};
  size_t off = 0;
  w.sig_rows = (uint16_t*)(base + off); off += al((size_t)d.n_tiles * 128 * d.Kp * 2);
  w.sig_cols = (uint16_t*)(base + off); off += al((size_t)d.n_chunks * 128 * d.KC * 2);
  w.bhi = (uint16_t*)(base + off); off += al((size_t)d.Np * d.Kp * 2);
  w.blo = (uint16_t*)(base + off); off += al((size_t)d.Np * d.Kp * 2);
  w.wsum = (double2*)(base + off); off += al((size_t)d.n_tiles * sizeof(double2));
  w.status = (int*)(base + off); off += al(sizeof(int) * 4);
  return w;
}

int tc_prepare_step(const TcDims& d, int64_t n_samples, const uint32_t* bits, const TcWork& w, cudaStream_t st) {
  QES_CUDA_CHECK(cudaMemsetAsync(w.status, 0, sizeof(int), st));
  tc_sigma_rows_kernel<<<592, 256, 0, st>>>(d.ns, d.Kp, n_samples, d.n_tiles, bits, w.sig_rows);
  QES_LAUNCH_CHECK();
  tc_sigma_cols_kernel<<<592, 256, 0, st>>>(d.ns, d.KC, n_samples, d.n_chunks, bits, w.sig_cols);
  QES_LAUNCH_CHECK();
  return QES_OK;
}

template <class T, class V>
static int tc_matvec_t(const TcDims& d, int64_t n_samples, const uint32_t* bits, const T* tt, const V* v,
                       float2* w_out, T* partial, const TcWork& w, cudaStream_t st) {
  QES_CUDA_CHECK(cudaFuncSetAttribute(tc_ov_kernel<T, V>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTcSmemLimit));
  QES_CUDA_CHECK(cudaFuncSetAttribute(tc_ohu_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTcSmemLimit));
  const bool cplx = ScalarTraits<T>::is_complex;
  const int items = d.Np * (d.Kp / 8);
  tc_build_v_kernel<V><<<(items + 255) / 256, 256, 0, st>>>(d.ns, d.nh, d.Kp, d.Mp, d.Np, cplx, v, w.bhi, w.blo);
  QES_LAUNCH_CHECK();
  tc_ov_kernel<T, V><<<d.n_tiles, kThreads, d.ov_smem, st>>>(d, n_samples, bits, tt, v, w.sig_rows, w.bhi, w.blo, w_out,
                                                           w.wsum, w.status);
  QES_LAUNCH_CHECK();
  tc_ohu_kernel<T><<<d.n_chunks, kThreads, d.ohu_smem, st>>>(d, n_samples, bits, tt, w_out, w.wsum, d.n_tiles,
                                                             1.0 / (double)n_samples, w.sig_cols, partial, w.status);
  QES_LAUNCH_CHECK();
  return QES_OK;
}

int tc_matvec(int dtype, const TcDims& d, int64_t n_samples, const uint32_t* bits, const void* tanh_theta,
              const void* v, float2* w_out, void* partial, const TcWork& w, cudaStream_t st) {
  if (dtype == QES_DTYPE_C64)
    return tc_matvec_t<float2, double2>(d, n_samples, bits, (const float2*)tanh_theta, (const double2*)v, w_out,
                                        (float2*)partial, w, st);
  return tc_matvec_t<float, double>(d, n_samples, bits, (const float*)tanh_theta, (const double*)v, w_out,
                                    (float*)partial, w, st);
}

// O^H ((g - [mean g]) * scale) alone (force / VJP): the ohu kernel with the caller's vector
int tc_ohu(int dtype, const TcDims& d, int64_t n_samples, const uint32_t* bits, const void* tanh_theta,
           const float2* g, const double2* gsum_part, int gsum_n, double scale, void* partial, const TcWork& w,
           cudaStream_t st) {
  if (dtype == QES_DTYPE_C64) {
    QES_CUDA_CHECK(cudaFuncSetAttribute(tc_ohu_kernel<float2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTcSmemLimit));
    tc_ohu_kernel<float2><<<d.n_chunks, kThreads, d.ohu_smem, st>>>(d, n_samples, bits, (const float2*)tanh_theta, g,
                                                                    gsum_part, gsum_n, scale, w.sig_cols,
                                                                    (float2*)partial, w.status);
  } else {
    QES_CUDA_CHECK(cudaFuncSetAttribute(tc_ohu_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTcSmemLimit));
    tc_ohu_kernel<float><<<d.n_chunks, kThreads, d.ohu_smem, st>>>(d, n_samples, bits, (const float*)tanh_theta, g,
                                                                   gsum_part, gsum_n, scale, w.sig_cols,
                                                                   (float*)partial, w.status);
  }
  QES_LAUNCH_CHECK();
  return QES_OK;
}
