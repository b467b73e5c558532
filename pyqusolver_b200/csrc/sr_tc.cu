// Tensor-core (tcgen05) halves of the structured SR matvec.
//
//   ov : Y = T V'^T  with A = T (128 samples x K hidden), B = V' (NB x K)          -> TMEM
//        (O v)_s = sum_{i<ns} sigma_si Y_si + Y_{s,ns} + sigma_s . va          (epilogue)
//        V' stacks, per site i, the K-row [Re V_i | -Im V_i] (-> Re Y) and
//        [Im V_i | Re V_i] (-> Im Y) over the K = [Re t | Im t] axis; the extra
//        "site" ns carries v_b, so t_s . v_b comes out of the same MMA.
//   ohu: G_W = Sigma^T Q  with A = Sigma^T (128 sites x KC samples),
//        B = Q^T (2 Mp x KC), Q_sm = conj(t_sm) u_s, u_s = (w_s - mean w) / Ns    -> TMEM
//
// Operands are stored in global memory as BF16 core-matrix tiles (K-major, no
// swizzle, see umma.cuh), prepared once per VMC step (T, T^T, Sigma^T) or once
// per CG iteration (V'), and move into shared memory only by bulk copies.  ov
// streams K in chunks through a 4-stage mbarrier pipeline (producer thread ->
// MMA-issuing thread -> producer); ohu bulk-copies T^T for its sample chunk
// and multiplies it by u in shared memory.
//
// Precision: Sigma (+-1) is exact in BF16; every other operand x is split as
// x = hi + lo (two BF16 terms); ov uses hi*hi + hi*lo + lo*hi, ohu rebuilds Q
// in float32 and splits it again.  Accumulation is FP32 in TMEM.
//
// Every mbarrier wait is bounded; on time-out the kernel records
// QES_ERR_TIMEOUT in *status, still waits (bounded) for the work it issued,
// frees its TMEM and returns.  The host reads *status after the solve.
#include "common.cuh"
#include "sr_tc.h"

#include <cooperative_groups.h>
#include "umma.cuh"

#include <algorithm>
#include <atomic>
#include <cuda_bf16.h>

namespace {

constexpr uint32_t kWaitLimit = 1u << 22;     // try_wait polls before giving up
constexpr int kThreads = 512;                  // 16 warps; warp w reads TMEM lane quarter w % 4
constexpr int kWarps = kThreads / 32;
constexpr int kColGroups = kWarps / 4;         // warps sharing one lane quarter split the columns

__device__ __forceinline__ uint16_t bf16_bits(float x) { return __bfloat16_as_ushort(__float2bfloat16_rn(x)); }
__device__ __forceinline__ float bf16_val(uint16_t b) { return __bfloat162float(__ushort_as_bfloat16(b)); }
__device__ __forceinline__ void split_bf16(float x, uint16_t& hi, uint16_t& lo) {
  hi = bf16_bits(x);
  lo = bf16_bits(x - bf16_val(hi));
}
// the same split for two values at once, packed as bf16x2 (first value in the low half)
__device__ __forceinline__ void split2_bf16(float x0, float x1, uint32_t& hi, uint32_t& lo) {
  const __nv_bfloat162 h = __floats2bfloat162_rn(x0, x1);
  const float2 hf = __bfloat1622float2(h);
  const __nv_bfloat162 l = __floats2bfloat162_rn(x0 - hf.x, x1 - hf.y);
  hi = *reinterpret_cast<const uint32_t*>(&h);
  lo = *reinterpret_cast<const uint32_t*>(&l);
}
__device__ __forceinline__ uint32_t pack2(uint16_t a, uint16_t b) { return (uint32_t)a | ((uint32_t)b << 16); }
__device__ __forceinline__ uint4 pack8(const uint16_t (&v)[8]) {
  return make_uint4(pack2(v[0], v[1]), pack2(v[2], v[3]), pack2(v[4], v[5]), pack2(v[6], v[7]));
}
__device__ __forceinline__ void unpack8(uint4 p, float (&v)[8]) {
  const uint32_t w[4] = {p.x, p.y, p.z, p.w};
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    v[2 * q] = bf16_val((uint16_t)(w[q] & 0xffffu));
    v[2 * q + 1] = bf16_val((uint16_t)(w[q] >> 16));
  }
}

__device__ __forceinline__ void record_error(int* status, int code) {
  if (status) atomicCAS(status, 0, code);
}

__device__ __forceinline__ float vre(const double* v, int64_t k) { return (float)v[k]; }
__device__ __forceinline__ float vre(const double2* v, int64_t k) { return (float)v[k].x; }
__device__ __forceinline__ float vim(const double*, int64_t) { return 0.f; }
__device__ __forceinline__ float vim(const double2* v, int64_t k) { return (float)v[k].y; }
__device__ __forceinline__ float tre(const float* t, int64_t k) { return t[k]; }
__device__ __forceinline__ float tre(const float2* t, int64_t k) { return t[k].x; }
__device__ __forceinline__ float tim(const float*, int64_t) { return 0.f; }
__device__ __forceinline__ float tim(const float2* t, int64_t k) { return t[k].y; }

}  // namespace

// ================================================================================================
// per-step operands
// ================================================================================================
// sig_cols: chunk c = 128 sites x samples [KC c, KC c + KC): Sigma^T, the ohu A operand.
// Row 127 (always beyond the last site) is all ones, so the same MMA yields g_b = sum_s Q_s.
__global__ void tc_sigma_cols_kernel(int ns, int KC, int64_t n_samples, int n_chunks, const uint32_t* __restrict__ bits,
                                     uint16_t* __restrict__ out) {
  const int nw = n_words(ns);
  const int64_t items = (int64_t)n_chunks * 128 * (KC / 8);
  for (int64_t it = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; it < items; it += (int64_t)gridDim.x * blockDim.x) {
    const int r = (int)(it % 128);                       // site (fastest: consecutive 16-byte stores)
    const int k8 = (int)((it / 128) % (KC / 8));
    const int64_t c = it / ((int64_t)(KC / 8) * 128);
    uint16_t v[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int64_t s = c * KC + 8 * k8 + q;
      v[q] = 0;
      if (s < n_samples && r < ns) v[q] = ((bits[s * nw + (r >> 5)] >> (r & 31)) & 1u) ? 0x3F80u : 0xBF80u;
      if (s < n_samples && r == 127) v[q] = 0x3F80u;      // row of ones: D[127] = sum_s Q_s = g_b
    }
    uint8_t* base = reinterpret_cast<uint8_t*>(out) + (size_t)c * 128 * KC * 2;
    *reinterpret_cast<uint4*>(base + umma::kmajor_offset(r, 8 * k8, 128)) = pack8(v);
  }
}

// t_rows: ov A operand.  Tile t (128 samples), chunk c of KCH columns of the K axis
// [Re t (Mp) | Im t (Mp)] (complex) or [t] (real), terms hi/lo:
//   byte offset ((t * nK + c) * 2 + term) * (128 * KCH * 2) + kmajor_offset(r, k % KCH, 128)
template <class T>
__global__ void tc_t_rows_kernel(TcDims d, int64_t n_samples, const T* __restrict__ tt, uint16_t* __restrict__ out) {
  constexpr bool CPLX = ScalarTraits<T>::is_complex;
  const int nh = d.nh, Kd = d.Kd, KCH = d.KCH, nK = Kd / KCH;
  const size_t tile_bytes = (size_t)128 * KCH * 2;
  const int64_t items = (int64_t)d.n_tiles * 128 * (Kd / 8);
  for (int64_t it = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; it < items; it += (int64_t)gridDim.x * blockDim.x) {
    const int r = (int)(it % 128);
    const int k8 = (int)((it / 128) % (Kd / 8));
    const int64_t t = it / ((int64_t)(Kd / 8) * 128);
    const int64_t s = t * 128 + r;
    uint16_t h[8], l[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int k = 8 * k8 + q;
      float x = 0.f;
      if (s < n_samples) {
        if (CPLX) {
          if (k < d.Mp) {
            if (k < nh) x = tre(tt, s * nh + k);
          } else if (k - d.Mp < nh) {
            x = tim(tt, s * nh + (k - d.Mp));
          }
        } else if (k < nh) {
          x = tre(tt, s * nh + k);
        }
      }
      split_bf16(x, h[q], l[q]);
    }
    const int c = (8 * k8) / KCH, kc = (8 * k8) % KCH;
    uint8_t* base = reinterpret_cast<uint8_t*>(out) + (((size_t)t * nK + c) * 2) * tile_bytes;
    const uint32_t off = umma::kmajor_offset(r, kc, 128);
    *reinterpret_cast<uint4*>(base + off) = pack8(h);
    *reinterpret_cast<uint4*>(base + tile_bytes + off) = pack8(l);
  }
}

// t_cols: ohu B operand before the u-scaling.  Chunk c (KC samples): rows n = hidden (re: n < Mp,
// im: Mp <= n < 2 Mp) x KC samples, terms hi/lo.
template <class T>
__global__ void tc_t_cols_kernel(TcDims d, int64_t n_samples, const T* __restrict__ tt, uint16_t* __restrict__ out) {
  constexpr bool CPLX = ScalarTraits<T>::is_complex;
  const int nh = d.nh, Mp = d.Mp, Np = d.Np, KC = d.KC;
  const size_t term_bytes = (size_t)Np * KC * 2;
  const int64_t items = (int64_t)d.n_chunks * Np * (KC / 8);
  for (int64_t it = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; it < items; it += (int64_t)gridDim.x * blockDim.x) {
    const int n = (int)(it % Np);
    const int k8 = (int)((it / Np) % (KC / 8));
    const int64_t c = it / ((int64_t)(KC / 8) * Np);
    const bool im = CPLX && n >= Mp;
    const int m = im ? n - Mp : n;
    uint16_t h[8], l[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int64_t s = c * KC + 8 * k8 + q;
      float x = 0.f;
      if (s < n_samples && m < nh) x = im ? tim(tt, s * nh + m) : tre(tt, s * nh + m);
      split_bf16(x, h[q], l[q]);
    }
    uint8_t* base = reinterpret_cast<uint8_t*>(out) + (size_t)c * 2 * term_bytes;
    const uint32_t off = umma::kmajor_offset(n, 8 * k8, Np);
    *reinterpret_cast<uint4*>(base + off) = pack8(h);
    *reinterpret_cast<uint4*>(base + term_bytes + off) = pack8(l);
  }
}

// ================================================================================================
// per-iteration operand of ov: V' (NB rows x Kd), chunked like t_rows:
//   byte offset (c * 2 + term) * (NB * KCH * 2) + kmajor_offset(n, k % KCH, NB)
// ================================================================================================
template <class V>
__global__ void tc_build_vp_kernel(TcDims d, bool cplx, const V* __restrict__ v, uint16_t* __restrict__ out) {
  pdl_trigger();
  pdl_wait();                                             // v comes from the previous kernel
  const int ns = d.ns, nh = d.nh, Mp = d.Mp, KCH = d.KCH, NB = d.NB, Sp = d.Sp;
  const bool spl = d.splitc;                               // V'': K = hidden units, rows Re v then Im v
  const V* vb = v + ns;
  const V* vW = v + ns + nh;
  const size_t term_bytes = (size_t)NB * KCH * 2;
  const int items = NB * (d.VK / 8);
  for (int it = blockIdx.x * blockDim.x + threadIdx.x; it < items; it += gridDim.x * blockDim.x) {
    const int n = it % NB, k8 = it / NB;
    const bool yim = cplx && n >= Sp;                     // row produces Im Y
    const int i = yim ? n - Sp : n;                        // site (i == ns: the v_b row)
    uint16_t h[8], l[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int k = 8 * k8 + q;
      const bool kim = !spl && cplx && k >= Mp;            // K column holds Im t
      const int m = kim ? k - Mp : k;
      float x = 0.f;
      if (m < nh && i <= ns) {
        const float vr = (i < ns) ? vre(vW, (int64_t)i * nh + m) : vre(vb, m);
        const float vi = (i < ns) ? vim(vW, (int64_t)i * nh + m) : vim(vb, m);
        // Re Y = Re t Re v - Im t Im v ;  Im Y = Re t Im v + Im t Re v
        if (spl) x = yim ? vi : vr;
        else if (!yim) x = kim ? -vi : vr;
        else x = kim ? vr : vi;
      }
      split_bf16(x, h[q], l[q]);
    }
    const int c = (8 * k8) / KCH, kc = (8 * k8) % KCH;
    uint8_t* base = reinterpret_cast<uint8_t*>(out) + (size_t)c * 2 * term_bytes;
    const uint32_t off = umma::kmajor_offset(n, kc, NB);
    *reinterpret_cast<uint4*>(base + off) = pack8(h);
    *reinterpret_cast<uint4*>(base + term_bytes + off) = pack8(l);
  }
}

// ov epilogue helpers.  wrd[128 w] is spin word w of the sample row (bit i % 32 of word i / 32 is
// site i, set = spin up).  spin_window(i0): bit q = spin of site i0 + q (i0 >= -31; sites below 0
// read as 0).  low_mask(c): the lowest c bits (c clamped to [0, 32]).
__device__ __forceinline__ uint32_t spin_window(const uint32_t* wrd, int nw, int i0) {
  if (i0 < 0) return wrd[0] << (-i0);
  const int w = i0 >> 5, sh = i0 & 31;
  const uint32_t lo = wrd[128 * w], hi = (w + 1 < nw) ? wrd[128 * (w + 1)] : 0u;
  return __funnelshift_r(lo, hi, sh);
}
__device__ __forceinline__ uint32_t low_mask(int c) {
  return c <= 0 ? 0u : (c >= 32 ? 0xffffffffu : ((1u << c) - 1u));
}
// fold 16 accumulator columns [n0, n0 + 16) of one sample row into (O v)_s: column n < Sp is
// (Re) Y of site n, n >= Sp (complex) is Im Y of site n - Sp; a site below ns with spin down
// flips the sign (a sign-bit xor), site ns (the v_b row) and the zero padding add as they are.
template <bool CPLX>
__device__ __forceinline__ void ov_fold16(int n0, const float (&y)[16], int ns, int Sp, const uint32_t* wrd, int nw,
                                          float2& acc) {
  const int nre = CPLX ? (Sp - n0) : 16;                  // columns of the real half in this group
  uint32_t neg = 0;
  if (nre > 0) neg |= ~spin_window(wrd, nw, n0) & low_mask(ns - n0) & low_mask(nre);
  if (CPLX && nre < 16) neg |= ~spin_window(wrd, nw, n0 - Sp) & low_mask(ns - (n0 - Sp)) & ~low_mask(nre);
  float sre = 0.f, sim = 0.f;
#pragma unroll
  for (int q = 0; q < 16; ++q) {
    const float v = __int_as_float(__float_as_int(y[q]) ^ (int)(((neg >> q) & 1u) << 31));
    if (!CPLX || q < nre) sre += v;
    else sim += v;
  }
  acc.x += sre;
  acc.y += sim;
}

// ================================================================================================
// ov: one CTA per 128-sample tile, K streamed through a d.ov_stages-deep pipeline
// ================================================================================================
template <class T, class V>
__global__ void __launch_bounds__(kThreads) tc_ov_kernel(TcDims d, int64_t n_samples, const uint32_t* __restrict__ bits,
                                                         const V* __restrict__ v, const uint16_t* __restrict__ t_rows,
                                                         const uint16_t* __restrict__ vp, float2* __restrict__ w_out,
                                                         double2* __restrict__ wsum_part, int* __restrict__ status,
                                                         const double* __restrict__ cg_done,
                                                         const float* __restrict__ wts) {
  extern __shared__ __align__(128) uint8_t smem[];
  constexpr bool CPLX = ScalarTraits<T>::is_complex;
  const int ns = d.ns, KCH = d.KCH, NB = d.NB, Sp = d.Sp;
  const int nK = d.Kd / KCH;                               // K chunks of a T tile
  // split-complex: a stage holds the Re t and Im t chunks of the same hidden units and one V'' chunk;
  // nKh = chunks per half (the Im chunks of a tile start there); the pipeline runs over nKh stages
  const bool spl = d.splitc;
  const int nKh = d.VK / KCH;
  const int nP = spl ? nKh : nK;
  const uint32_t a_term = 128u * KCH * 2u, b_term = (uint32_t)NB * KCH * 2u;
  const uint32_t a_bytes = (spl ? 4u : 2u) * a_term;       // A part of a stage (hi, lo[, Im hi, Im lo])
  const uint32_t stage_bytes = a_bytes + 2u * b_term;
  const int S = d.ov_stages;
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + S * stage_bytes);
  uint64_t* empty = full + S;
  uint64_t* done = empty + S;
  uint32_t* tslot = reinterpret_cast<uint32_t*>(done + 1);
  T* s_va = reinterpret_cast<T*>(tslot + 4);
  const int nw = n_words(ns);
  // spin words of the tile, word-major ([word][row]) so that a warp reads consecutive rows
  uint32_t* s_bits = reinterpret_cast<uint32_t*>(reinterpret_cast<uint8_t*>(s_va) +
                                                 (((size_t)ns * sizeof(T) + 15) & ~(size_t)15));
  __shared__ double2 red[4];
  __shared__ float2 s_part[kColGroups][128];

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int tile = blockIdx.x;
  const uint8_t* ga = reinterpret_cast<const uint8_t*>(t_rows) + (size_t)tile * nK * 2 * a_term;
  const uint8_t* gb = reinterpret_cast<const uint8_t*>(vp);
  pdl_trigger();
  if (cg_block_done(cg_done)) {         // converged CG: nothing issued yet, nothing to drain
    pdl_wait();
    return;
  }
  if (tid == 0) {
    for (int q = 0; q < S; ++q) {
      umma::mbar_init(&full[q], 1);
      umma::mbar_init(&empty[q], 1);
    }
    umma::mbar_init(done, 1);
    umma::fence_mbar_init();
    // the first S stages go out before the TMEM allocation and the block-wide setup; the T tiles
    // (per-step operands) even before the previous kernel, which writes V', has completed
    for (int c = 0; c < S && c < nP; ++c) {
      umma::mbar_arrive_expect_tx(&full[c], stage_bytes);
      umma::bulk_g2s(smem + c * stage_bytes, ga + (size_t)c * 2 * a_term, 2 * a_term, &full[c]);
      if (spl)
        umma::bulk_g2s(smem + c * stage_bytes + 2 * a_term, ga + (size_t)(nKh + c) * 2 * a_term, 2 * a_term,
                       &full[c]);
    }
  }
  pdl_wait();
  if (tid == 0) {
    for (int c = 0; c < S && c < nP; ++c)
      umma::bulk_g2s(smem + c * stage_bytes + a_bytes, gb + (size_t)c * 2 * b_term, 2 * b_term, &full[c]);
  }
  if (warp == 0) {
    umma::tmem_alloc(tslot, d.tmem_cols);
    umma::tmem_relinquish();
  }
  umma::tc_fence_before();
  __syncthreads();
  umma::tc_fence_after();
  const uint32_t tbase = *tslot;

  if (warp >= 2) {
    // while the pipeline runs: v_a and the tile's spin words into shared memory (epilogue inputs)
    const int t2 = tid - 64, n2 = kThreads - 64;
    for (int i = t2; i < ns; i += n2) {
      if constexpr (CPLX) s_va[i] = make_float2(vre(v, i), vim(v, i));
      else s_va[i] = vre(v, i);
    }
    const int64_t r0 = (int64_t)tile * 128;
    const int rows = (n_samples - r0 < 128) ? (int)(n_samples - r0) : 128;
    for (int q = t2; q < 128 * nw; q += n2) {
      const int r = q / nw, w = q - r * nw;
      s_bits[w * 128 + r] = (r < rows) ? bits[r0 * nw + q] : 0u;
    }
  } else if (warp == 0 && lane == 0) {
    // producer: stage s is refilled once the MMAs that read it have completed
    for (int c = S; c < nP; ++c) {
      const int s = c % S;
      if (!umma::mbar_wait(&empty[s], ((c / S) - 1) & 1, kWaitLimit)) {
        record_error(status, QES_ERR_TIMEOUT);
        break;
      }
      uint8_t* st = smem + s * stage_bytes;
      umma::mbar_arrive_expect_tx(&full[s], stage_bytes);
      umma::bulk_g2s(st, ga + (size_t)c * 2 * a_term, 2 * a_term, &full[s]);
      if (spl) umma::bulk_g2s(st + 2 * a_term, ga + (size_t)(nKh + c) * 2 * a_term, 2 * a_term, &full[s]);
      umma::bulk_g2s(st + a_bytes, gb + (size_t)c * 2 * b_term, 2 * b_term, &full[s]);
    }
  } else if (warp == 1 && lane == 0) {
    // MMA issuer: D (128 x NB) += A_hi B_hi + A_hi B_lo + A_lo B_hi over every 16-wide k-step;
    // NB > 256 is issued as two N parts (rows [0, 256) and [256, NB) of V') into adjacent TMEM columns
    // split-complex: D1 (columns 0..) += T_re V''^T, D2 (columns 256..) += T_im V''^T, three terms each
    const int n_parts = NB > 256 ? 2 : 1;
    const uint32_t np0 = NB > 256 ? 256u : (uint32_t)NB;
    for (int c = 0; c < nP; ++c) {
      const int s = c % S;
      if (!umma::mbar_wait(&full[s], (c / S) & 1, kWaitLimit)) {
        record_error(status, QES_ERR_TIMEOUT);
        break;
      }
      umma::tc_fence_after();
      const uint32_t sa = umma::smem_u32(smem + s * stage_bytes);
      const uint32_t ahi = sa, alo = sa + a_term, bhi = sa + a_bytes, blo = bhi + b_term;
      for (int kk = 0; kk < KCH / 16; ++kk) {
        const uint32_t ko_a = 2u * kk * 128u * 16u, ko_b = 2u * kk * NB * 16u;
        const uint64_t dah = umma::smem_desc(ahi + ko_a, 128u * 16u, 128u);
        const uint64_t dal = umma::smem_desc(alo + ko_a, 128u * 16u, 128u);
        if (spl) {
          const uint32_t idesc = umma::idesc_bf16_f32(128, (uint32_t)NB);
          const uint64_t dih = umma::smem_desc(ahi + 2 * a_term + ko_a, 128u * 16u, 128u);
          const uint64_t dil = umma::smem_desc(ahi + 3 * a_term + ko_a, 128u * 16u, 128u);
          const uint64_t dbh = umma::smem_desc(bhi + ko_b, NB * 16u, 128u);
          const uint64_t dbl = umma::smem_desc(blo + ko_b, NB * 16u, 128u);
          const uint32_t acc = (c > 0 || kk > 0) ? 1u : 0u;
          umma::mma_bf16(tbase, dah, dbh, idesc, acc);
          umma::mma_bf16(tbase, dah, dbl, idesc, 1u);
          umma::mma_bf16(tbase, dal, dbh, idesc, 1u);
          umma::mma_bf16(tbase + 256u, dih, dbh, idesc, acc);
          umma::mma_bf16(tbase + 256u, dih, dbl, idesc, 1u);
          umma::mma_bf16(tbase + 256u, dil, dbh, idesc, 1u);
          continue;
        }
        for (int pt = 0; pt < n_parts; ++pt) {
          const uint32_t n0 = pt ? np0 : 0u, nn = pt ? (uint32_t)NB - np0 : np0;
          const uint32_t idesc = umma::idesc_bf16_f32(128, nn);
          const uint32_t rb = (n0 / 8u) * 128u;        // first 8-row group of this part
          const uint64_t dbh = umma::smem_desc(bhi + ko_b + rb, NB * 16u, 128u);
          const uint64_t dbl = umma::smem_desc(blo + ko_b + rb, NB * 16u, 128u);
          umma::mma_bf16(tbase + n0, dah, dbh, idesc, (c > 0 || kk > 0) ? 1u : 0u);
          umma::mma_bf16(tbase + n0, dah, dbl, idesc, 1u);
          umma::mma_bf16(tbase + n0, dal, dbh, idesc, 1u);
        }
      }
      umma::mma_commit(&empty[s]);
    }
    umma::mma_commit(done);                 // arrives once every MMA issued above has completed
  }
  __syncthreads();
  if (!umma::mbar_wait(done, 0, kWaitLimit)) record_error(status, QES_ERR_TIMEOUT);
  umma::tc_fence_after();

  // epilogue: warp w reads lane quarter w % 4 (sample rows) and column group w / 4
  const int quarter = warp & 3, cg = warp >> 2;
  const int row = 32 * quarter + lane;
  const int64_t s = (int64_t)tile * 128 + row;
  const bool sval = s < n_samples;
  const uint32_t* wrd = s_bits + row;                     // word w of this row at wrd[128 w]
  float2 acc = make_float2(0.f, 0.f);
  const uint32_t lane_addr = tbase + ((uint32_t)(32 * quarter) << 16);
  int c = cg;
  // two column groups per TMEM wait
  for (; c + kColGroups < NB / 16; c += 2 * kColGroups) {
    float y0[16], y1[16];
    umma::tmem_ld16x2(lane_addr + 16 * c, lane_addr + 16 * (c + kColGroups), y0, y1);
    ov_fold16<CPLX>(16 * c, y0, ns, Sp, wrd, nw, acc);
    ov_fold16<CPLX>(16 * (c + kColGroups), y1, ns, Sp, wrd, nw, acc);
  }
  if (c < NB / 16) {
    float y[16];
    umma::tmem_ld16(lane_addr + 16 * c, y);
    ov_fold16<CPLX>(16 * c, y, ns, Sp, wrd, nw, acc);
  }
  if (spl) {
    // D2 = T_im V''^T: column n < Sp is Im t . Re v_n (-> Im Y_n), column Sp + n is Im t . Im v_n
    // (-> -Re Y_n); folded with the same spin signs, then rotated into acc
    float2 acc2 = make_float2(0.f, 0.f);
    for (int c2 = cg; c2 < NB / 16; c2 += kColGroups) {
      float y[16];
      umma::tmem_ld16(lane_addr + 256u + 16 * c2, y);
      ov_fold16<CPLX>(16 * c2, y, ns, Sp, wrd, nw, acc2);
    }
    acc.x -= acc2.y;
    acc.y += acc2.x;
  }
  // + sigma_s . v_a: column group cg takes the sites of spin words cg, cg + 4, ...
  for (int w = cg; w < nw; w += kColGroups) {
    const uint32_t word = wrd[128 * w];
    const int i1 = (32 * w + 32 < ns) ? 32 * w + 32 : ns;
    float sre = 0.f, sim = 0.f;
    for (int i = 32 * w; i < i1; ++i) {
      const int sgn = (int)((~word >> (i & 31)) & 1u) << 31;
      const T va = s_va[i];
      if constexpr (CPLX) {
        sre += __int_as_float(__float_as_int(va.x) ^ sgn);
        sim += __int_as_float(__float_as_int(va.y) ^ sgn);
      } else {
        sre += __int_as_float(__float_as_int(va) ^ sgn);
      }
    }
    acc.x += sre;
    acc.y += sim;
  }
  s_part[cg][row] = acc;
  umma::tc_fence_before();
  __syncthreads();
  if (cg == 0) {
    float2 wv = s_part[0][row];
#pragma unroll
    for (int g = 1; g < kColGroups; ++g) wv = wv + s_part[g][row];
    if (!sval) wv = make_float2(0.f, 0.f);
    if (sval) w_out[s] = wv;
    const double wt = (wts && sval) ? (double)wts[s] : 1.0;          // weighted sum for the weighted mean
    double2 ps = make_double2(wt * wv.x, wt * wv.y);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      ps.x += __shfl_xor_sync(0xffffffffu, ps.x, o);
      ps.y += __shfl_xor_sync(0xffffffffu, ps.y, o);
    }
    if (lane == 0) red[quarter] = ps;
  }
  __syncthreads();
  if (tid == 0) {
    double2 t = make_double2(0.0, 0.0);
    for (int q = 0; q < 4; ++q) { t.x += red[q].x; t.y += red[q].y; }
    wsum_part[tile] = t;
  }
  if (warp == 0) umma::tmem_dealloc(tbase, d.tmem_cols);
}

// ================================================================================================
// ovz: O v through z = Sigma V.  A = [sigma_s | 1] (128 samples x Kz: sites, the ones column at
// K index ns, zeros beyond), built by the CTA from the spin words, exact in BF16; B = Bz (hi/lo),
// NZ rows x Kz, copied whole into shared memory with one mbarrier per 16-wide k-step.  The MMAs
// give z_s = sigma_s^T V + v_b for every hidden unit (columns m: Re, Mp + m: Im) in TMEM, and the
// epilogue forms (O v)_s = sum_m t_sm z_sm + sigma_s . v_a with t in float32, read from T transposed
// per 128-sample tile once per step (t_tiles[tile][m][row]: the 32 rows of a warp are 32 consecutive
// elements).  Against tc_ov_kernel: K is the sites (Kz = 112 for 100 sites) instead of the hidden
// axis (2 Mp = 416 complex), and only B is split, so a tile takes two MMAs per k-step instead of
// three per K column pair.
// ================================================================================================
// T per 128-sample tile, transposed: out[tile][m][r] = T[tile * 128 + r][m] (rows beyond Ns: 0).
// Block (32 x 8) moves a 32 x 32 (rows x units) square through shared memory.
template <class T>
__global__ void tc_t_tiles_kernel(int nh, int64_t n_samples, int n_tiles, const T* __restrict__ tt,
                                  T* __restrict__ out) {
  __shared__ T sq[32][33];
  const int mb = (nh + 31) / 32;
  const int64_t squares = (int64_t)n_tiles * 4 * mb;
  for (int64_t q = blockIdx.x; q < squares; q += gridDim.x) {
    const int m0 = 32 * (int)(q % mb);
    const int64_t rq = q / mb;                             // 32-row block of the whole sample range
    const int64_t r0 = 32 * rq;
    __syncthreads();
    for (int i = threadIdx.y; i < 32; i += 8) {
      const int64_t s = r0 + i;
      const int m = m0 + threadIdx.x;
      sq[i][threadIdx.x] = (s < n_samples && m < nh) ? tt[s * nh + m] : ScalarTraits<T>::zero();
    }
    __syncthreads();
    const int64_t tile = rq >> 2;
    const int rr = (int)(rq & 3) * 32 + threadIdx.x;      // row within the tile
    for (int j = threadIdx.y; j < 32; j += 8) {
      const int m = m0 + j;
      if (m < nh) out[((size_t)tile * nh + m) * 128 + rr] = sq[threadIdx.x][j];
    }
  }
}

// Bz operand from the direction vector v (v_a, v_b, W row-major [site][hidden unit]):
// item (n, k8) writes the 8 K entries [8 k8, 8 k8 + 8) of row n, hi and lo
template <class V>
__global__ void tc_build_vz_kernel(TcDims d, bool cplx, const V* __restrict__ v, uint16_t* __restrict__ out) {
  pdl_trigger();
  pdl_wait();                                             // v comes from the previous kernel
  const int ns = d.ns, nh = d.nh, Mp = d.Mp, NZ = d.NZ;
  const V* vb = v + ns;
  const V* vW = v + ns + nh;
  const size_t tile_bytes = (size_t)NZ * 32;
  const int items = NZ * (d.Kz / 8);
  for (int it = blockIdx.x * blockDim.x + threadIdx.x; it < items; it += gridDim.x * blockDim.x) {
    const int n = it % NZ, k8 = it / NZ;
    const bool im = cplx && n >= Mp;
    const int m = im ? n - Mp : n;
    uint16_t h[8], l[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int k = 8 * k8 + q;                           // site (k == ns: v_b)
      float x = 0.f;
      if (m < nh && k <= ns) {
        if (k < ns) x = im ? vim(vW, (int64_t)k * nh + m) : vre(vW, (int64_t)k * nh + m);
        else x = im ? vim(vb, m) : vre(vb, m);
      }
      split_bf16(x, h[q], l[q]);
    }
    uint8_t* base = reinterpret_cast<uint8_t*>(out) + (size_t)(k8 >> 1) * 2 * tile_bytes;
    const uint32_t off = umma::kmajor_offset(n, 8 * (k8 & 1), NZ);
    *reinterpret_cast<uint4*>(base + off) = pack8(h);
    *reinterpret_cast<uint4*>(base + tile_bytes + off) = pack8(l);
  }
}

// t of 16 hidden units [m0, m0 + 16) of one sample row from the tile-transposed T (element (m, r)
// at tcol[m * 128]: a warp's 32 rows read 32 consecutive elements), zero beyond nh
template <class T>
__device__ __forceinline__ void ovz_load16(const T* __restrict__ tcol, int m0, int nh, T (&t)[16]) {
#pragma unroll
  for (int q = 0; q < 16; ++q) t[q] = (m0 + q < nh) ? __ldg(tcol + (size_t)(m0 + q) * 128) : ScalarTraits<T>::zero();
}
__device__ __forceinline__ void ovz_dot16(const float2 (&t)[16], const float (&zr)[16], const float (&zi)[16],
                                          float2& acc) {
  float ar = 0.f, ai = 0.f;
#pragma unroll
  for (int q = 0; q < 16; ++q) {
    ar = fmaf(t[q].x, zr[q], fmaf(-t[q].y, zi[q], ar));
    ai = fmaf(t[q].x, zi[q], fmaf(t[q].y, zr[q], ai));
  }
  acc.x += ar;
  acc.y += ai;
}
__device__ __forceinline__ void ovz_dot16(const float (&t)[16], const float (&zr)[16], const float (&)[16],
                                          float2& acc) {
  float a = 0.f;
#pragma unroll
  for (int q = 0; q < 16; ++q) a = fmaf(t[q], zr[q], a);
  acc.x += a;
}

template <class T, class V>
__global__ void __launch_bounds__(kThreads) tc_ovz_kernel(TcDims d, int64_t n_samples, const uint32_t* __restrict__ bits,
                                                          const V* __restrict__ v, const T* __restrict__ t_tiles,
                                                          const uint16_t* __restrict__ vz, float2* __restrict__ w_out,
                                                          double2* __restrict__ wsum_part, int* __restrict__ status,
                                                          const double* __restrict__ cg_done,
                                                          const float* __restrict__ wts) {
  extern __shared__ __align__(128) uint8_t smem[];
  constexpr bool CPLX = ScalarTraits<T>::is_complex;
  const int ns = d.ns, nh = d.nh, Kz = d.Kz, NZ = d.NZ, Mp = d.Mp;
  const int nks = Kz / 16;
  const uint32_t a_bytes = 128u * Kz * 2u;
  const uint32_t ks_bytes = 2u * NZ * 32u;                 // one k-step of Bz: hi and lo tiles
  uint8_t* sA = smem;
  uint8_t* sB = smem + a_bytes;
  uint64_t* full = reinterpret_cast<uint64_t*>(sB + (size_t)nks * ks_bytes);
  uint64_t* done = full + nks;
  uint32_t* tslot = reinterpret_cast<uint32_t*>(done + 1);
  T* s_va = reinterpret_cast<T*>(tslot + 4);
  const int nw = n_words(ns);
  // spin words of the tile, word-major ([word][row]) so that a warp reads consecutive rows
  uint32_t* s_bits = reinterpret_cast<uint32_t*>(reinterpret_cast<uint8_t*>(s_va) +
                                                 (((size_t)ns * sizeof(T) + 15) & ~(size_t)15));
  __shared__ double2 red[4];
  __shared__ float2 s_part[kColGroups][128];

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int tile = blockIdx.x;
  pdl_trigger();
  if (cg_block_done(cg_done)) {         // converged CG: nothing issued yet, nothing to drain
    pdl_wait();
    return;
  }
  if (tid == 0) {
    for (int c = 0; c < nks; ++c) umma::mbar_init(&full[c], 1);
    umma::mbar_init(done, 1);
    umma::fence_mbar_init();
    // the tile's transposed T (per-step data, read in the epilogue) is pulled into L2 while this
    // CTA waits on its predecessor
    const size_t tbytes = (size_t)nh * 128 * sizeof(T);
    if (d.prefetch && ((reinterpret_cast<uintptr_t>(t_tiles) | tbytes) & 15) == 0) {
      const uint8_t* tb = reinterpret_cast<const uint8_t*>(t_tiles) + (size_t)tile * tbytes;
      for (size_t o = 0; o < tbytes; o += 65536)
        umma::bulk_prefetch_l2(tb + o, (uint32_t)((tbytes - o < 65536) ? (tbytes - o) : 65536));
    }
  }
  // per-step inputs (older than the previous kernel): the tile's spin words, then A
  const int64_t r0 = (int64_t)tile * 128;
  const int rows = (n_samples - r0 < 128) ? (int)(n_samples - r0) : 128;
  for (int q = tid; q < 128 * nw; q += kThreads) {
    const int r = q / nw, w = q - r * nw;
    s_bits[w * 128 + r] = (r < rows) ? bits[r0 * nw + q] : 0u;
  }
  __syncthreads();
  for (int it = tid; it < 128 * (Kz / 8); it += kThreads) {
    const int r = it & 127, k8 = it >> 7;
    uint16_t a[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int k = 8 * k8 + q;
      uint16_t x = 0;
      if (r < rows) {
        if (k < ns) x = ((s_bits[(k >> 5) * 128 + r] >> (k & 31)) & 1u) ? 0x3F80u : 0xBF80u;
        else if (k == ns) x = 0x3F80u;                    // the v_b column
      }
      a[q] = x;
    }
    *reinterpret_cast<uint4*>(sA + umma::kmajor_offset(r, 8 * k8, 128)) = pack8(a);
  }
  umma::fence_proxy_async_smem();       // A (generic-proxy stores) -> visible to the tensor core
  pdl_wait();                           // Bz and v_a: written by the previous kernel
  if (tid == 0) {
    for (int c = 0; c < nks; ++c) {
      umma::mbar_arrive_expect_tx(&full[c], ks_bytes);
      umma::bulk_g2s(sB + (size_t)c * ks_bytes, reinterpret_cast<const uint8_t*>(vz) + (size_t)c * ks_bytes, ks_bytes,
                     &full[c]);
    }
  }
  for (int i = tid; i < ns; i += kThreads) {
    if constexpr (CPLX) s_va[i] = make_float2(vre(v, i), vim(v, i));
    else s_va[i] = vre(v, i);
  }
  if (warp == 0) {
    umma::tmem_alloc(tslot, d.ovz_tmem);
    umma::tmem_relinquish();
  }
  umma::tc_fence_before();
  __syncthreads();
  umma::tc_fence_after();
  const uint32_t tbase = *tslot;

  // epilogue rows: warp w reads lane quarter w % 4 (sample rows) and column group w / 4
  const int quarter = warp & 3, cg = warp >> 2;
  const int row = 32 * quarter + lane;
  const int64_t s = r0 + row;
  const bool sval = s < n_samples;
  const T* tcol = t_tiles + (size_t)tile * nh * 128 + row;
  const uint32_t* wrd = s_bits + row;                     // word w of this row at wrd[128 w]
  float2 acc = make_float2(0.f, 0.f);
  // sigma_s . v_a first (column group cg takes spin words cg, cg + 4, ...), while Bz is in flight
  for (int w = cg; w < nw; w += kColGroups) {
    const uint32_t word = wrd[128 * w];
    const int i1 = (32 * w + 32 < ns) ? 32 * w + 32 : ns;
    float sre = 0.f, sim = 0.f;
    for (int i = 32 * w; i < i1; ++i) {
      const int sgn = (int)((~word >> (i & 31)) & 1u) << 31;
      const T va = s_va[i];
      if constexpr (CPLX) {
        sre += __int_as_float(__float_as_int(va.x) ^ sgn);
        sim += __int_as_float(__float_as_int(va.y) ^ sgn);
      } else {
        sre += __int_as_float(__float_as_int(va) ^ sgn);
      }
    }
    acc.x += sre;
    acc.y += sim;
  }
  if (warp == 1) {
    if (lane == 0) {
      // D (128 x NZ) = A Bz_hi^T + A Bz_lo^T; NZ > 256 is issued as two N parts
      const int n_parts = NZ > 256 ? 2 : 1;
      const uint32_t np0 = NZ > 256 ? 256u : (uint32_t)NZ;
      const uint32_t sa = umma::smem_u32(sA), sb = umma::smem_u32(sB);
      for (int c = 0; c < nks; ++c) {
        if (!umma::mbar_wait(&full[c], 0, kWaitLimit)) {
          record_error(status, QES_ERR_TIMEOUT);
          break;
        }
        umma::tc_fence_after();
        const uint64_t ad = umma::smem_desc(sa + (uint32_t)c * 2u * 128u * 16u, 128u * 16u, 128u);
        for (int pt = 0; pt < n_parts; ++pt) {
          const uint32_t n0 = pt ? np0 : 0u, nn = pt ? (uint32_t)NZ - np0 : np0;
          const uint32_t idesc = umma::idesc_bf16_f32(128, nn);
          const uint32_t bh = sb + (uint32_t)c * ks_bytes + (n0 / 8u) * 128u;
          const uint64_t dbh = umma::smem_desc(bh, (uint32_t)NZ * 16u, 128u);
          const uint64_t dbl = umma::smem_desc(bh + (uint32_t)NZ * 32u, (uint32_t)NZ * 16u, 128u);
          umma::mma_bf16(tbase + n0, ad, dbh, idesc, c > 0 ? 1u : 0u);
          umma::mma_bf16(tbase + n0, ad, dbl, idesc, 1u);
        }
      }
      umma::mma_commit(done);               // arrives once every MMA issued above has completed
    }
    __syncwarp();
  }
  // t of the first 16-unit chunk is loaded before the MMAs complete; each pass loads the next
  const uint32_t lane_addr = tbase + ((uint32_t)(32 * quarter) << 16);
  const int nch = (nh + 15) / 16;
  T tcur[16];
  if (cg < nch) ovz_load16(tcol, 16 * cg, nh, tcur);
  if (!umma::mbar_wait(done, 0, kWaitLimit)) record_error(status, QES_ERR_TIMEOUT);
  umma::tc_fence_after();
  for (int c = cg; c < nch; c += kColGroups) {
    T tnext[16];
    if (c + kColGroups < nch) ovz_load16(tcol, 16 * (c + kColGroups), nh, tnext);
    float zr[16], zi[16];
    if constexpr (CPLX) umma::tmem_ld16x2(lane_addr + 16 * c, lane_addr + Mp + 16 * c, zr, zi);
    else umma::tmem_ld16(lane_addr + 16 * c, zr);
    ovz_dot16(tcur, zr, zi, acc);
#pragma unroll
    for (int q = 0; q < 16; ++q) tcur[q] = tnext[q];
  }
  s_part[cg][row] = acc;
  umma::tc_fence_before();
  __syncthreads();
  if (cg == 0) {
    float2 wv = s_part[0][row];
#pragma unroll
    for (int g = 1; g < kColGroups; ++g) wv = wv + s_part[g][row];
    if (!sval) wv = make_float2(0.f, 0.f);
    if (sval) w_out[s] = wv;
    const double wt = (wts && sval) ? (double)wts[s] : 1.0;          // weighted sum for the weighted mean
    double2 ps = make_double2(wt * wv.x, wt * wv.y);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      ps.x += __shfl_xor_sync(0xffffffffu, ps.x, o);
      ps.y += __shfl_xor_sync(0xffffffffu, ps.y, o);
    }
    if (lane == 0) red[quarter] = ps;
  }
  __syncthreads();
  if (tid == 0) {
    double2 t = make_double2(0.0, 0.0);
    for (int q = 0; q < 4; ++q) { t.x += red[q].x; t.y += red[q].y; }
    wsum_part[tile] = t;
    // a k-step whose wait gave up may still be in flight: drain every copy (bounded) before exit
    for (int c = 0; c < nks; ++c) umma::mbar_wait(&full[c], 0, kWaitLimit);
  }
  if (warp == 0) umma::tmem_dealloc(tbase, d.ovz_tmem);
}

// ================================================================================================
// ohu: one CTA per KC-sample chunk; writes one P-vector of partial sums
// ================================================================================================
// CL = 2: the CTAs run in clusters of two (chunks 2c, 2c + 1); after staging, each adds its half
// of the rows of both CTAs' partials through distributed shared memory and writes one partial per
// pair, so the split-K partials that go through L2 and the reduction are halved.
template <class T, int CL>
__global__ void __launch_bounds__(kThreads) tc_ohu_kernel(TcDims d, int64_t n_samples, const float2* __restrict__ w,
                                                          const double2* __restrict__ wsum_part, int wsum_n,
                                                          double scale, const uint16_t* __restrict__ sig_cols,
                                                          const uint16_t* __restrict__ t_cols, T* __restrict__ partial,
                                                          int* __restrict__ status, const double* __restrict__ cg_done,
                                                          const float* __restrict__ wts) {
  extern __shared__ __align__(128) uint8_t smem[];
  constexpr bool CPLX = ScalarTraits<T>::is_complex;
  const int ns = d.ns, nh = d.nh, Mp = d.Mp, Np = d.Np, KC = d.KC;
  const uint32_t a_bytes = 128u * KC * 2u, b_term = (uint32_t)Np * KC * 2u;
  uint8_t* sA = smem;
  uint8_t* sBh = sA + a_bytes;
  uint8_t* sBl = sBh + b_term;
  T* s_u = reinterpret_cast<T*>(sBl + b_term);            // KC
  T* s_gb = s_u + KC;                                      // nh (g_b staging, CL = 2)
  T* s_ga = s_gb + nh;                                     // ns (g_a staging, CL = 2)
  uint64_t* bars = reinterpret_cast<uint64_t*>(reinterpret_cast<uint8_t*>(s_ga + ns) +
                                               ((16 - (reinterpret_cast<uintptr_t>(s_ga + ns) & 15)) & 15));
  uint32_t* tslot = reinterpret_cast<uint32_t*>(bars + 2);
  __shared__ double2 s_mean;
  __shared__ int s_issued;

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int chunk = blockIdx.x;
  const bool valid = chunk < d.n_chunks;                  // CL = 2 pads the grid to an even size
  pdl_trigger();
  // converged CG: single CTAs leave at once (the pairs of CL = 2 must stay together, so they run)
  if (CL == 1 && cg_block_done(cg_done)) {
    pdl_wait();
    return;
  }
  const int64_t s0 = (int64_t)chunk * KC;
  const int64_t P = (int64_t)ns + nh + (int64_t)ns * nh;
  __shared__ double2 s_red[kWarps];
  if (tid == 0) {
    umma::mbar_init(&bars[0], 1);
    umma::mbar_init(&bars[1], 1);
    umma::fence_mbar_init();
    s_issued = 0;
    // operands first (per-step tiles, older than the previous kernel): the copy overlaps the
    // previous kernel's tail, the mean and the TMEM allocation
    if (valid) {
      umma::mbar_arrive_expect_tx(&bars[0], a_bytes + 2 * b_term);
      umma::bulk_g2s(sA, reinterpret_cast<const uint8_t*>(sig_cols) + (size_t)chunk * a_bytes, a_bytes, &bars[0]);
      umma::bulk_g2s(sBh, reinterpret_cast<const uint8_t*>(t_cols) + (size_t)chunk * 2 * b_term, 2 * b_term,
                     &bars[0]);
    }
  }
  pdl_wait();                                             // w and its partial sums: previous kernel
  // this thread's sample of w (and weight) is requested before the mean's block reduction, so the
  // two global round trips overlap (KC <= 256 < kThreads, tc_plan: one sample per thread)
  static_assert(kThreads >= 256, "one sample of the O^H u chunk per thread");
  float2 w_pre = make_float2(0.f, 0.f);
  float wt_pre = 1.f;
  if (tid < KC && s0 + tid < n_samples) {
    w_pre = w[s0 + tid];
    if (wts) wt_pre = wts[s0 + tid];
  }
  // mean of w: the per-tile partial sums are reduced by the whole block (fixed order)
  {
    double2 t = make_double2(0.0, 0.0);
    if (wsum_part && wsum_n > 0)
      for (int q = tid; q < wsum_n; q += kThreads) { t.x += wsum_part[q].x; t.y += wsum_part[q].y; }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      t.x += __shfl_xor_sync(0xffffffffu, t.x, o);
      t.y += __shfl_xor_sync(0xffffffffu, t.y, o);
    }
    if (lane == 0) s_red[warp] = t;
    __syncthreads();
    if (tid == 0) {
      double2 m = make_double2(0.0, 0.0);
      if (wsum_part && wsum_n > 0) {
        for (int q = 0; q < kWarps; ++q) { m.x += s_red[q].x; m.y += s_red[q].y; }
        m.x /= (double)n_samples;
        m.y /= (double)n_samples;
      } else if (wsum_part) {
        m = wsum_part[0];            // the mean itself
      }
      s_mean = m;
    }
  }
  if (warp == 0) {
    umma::tmem_alloc(tslot, d.tmem_cols);
    umma::tmem_relinquish();
  }
  umma::tc_fence_before();
  __syncthreads();
  umma::tc_fence_after();
  const uint32_t tbase = *tslot;
  const float mr = (float)s_mean.x, mi = (float)s_mean.y, fs = (float)scale;
  if (tid < KC) {
    T u = ScalarTraits<T>::zero();
    if (s0 + tid < n_samples) {
      const float f = wts ? fs * wt_pre : fs;
      if constexpr (CPLX) u = make_float2((w_pre.x - mr) * f, (w_pre.y - mi) * f);
      else u = (w_pre.x - mr) * f;
    }
    s_u[tid] = u;
  }
  __syncthreads();
  const bool loaded = valid && umma::mbar_wait(&bars[0], 0, kWaitLimit);
  if (valid && !loaded) record_error(status, QES_ERR_TIMEOUT);
  // Q = conj(t) u in place: item (m, k8) = rows m (re) and Mp + m (im) for 8 samples
  const int items = Mp * (KC / 8);
  int m = tid % Mp, k8 = tid / Mp;                        // item it = k8 * Mp + m, stepped by kThreads
  const int dm = kThreads % Mp, dk = kThreads / Mp;
  for (int it = tid; loaded && it < items; it += kThreads) {
    const uint32_t offr = umma::kmajor_offset(m, 8 * k8, Np);
    float trh[8], trl[8], tih[8], til[8];
    unpack8(*reinterpret_cast<const uint4*>(sBh + offr), trh);
    unpack8(*reinterpret_cast<const uint4*>(sBl + offr), trl);
    uint32_t offi = 0;
    if constexpr (CPLX) {
      offi = umma::kmajor_offset(Mp + m, 8 * k8, Np);
      unpack8(*reinterpret_cast<const uint4*>(sBh + offi), tih);
      unpack8(*reinterpret_cast<const uint4*>(sBl + offi), til);
    }
    uint32_t rh[4], rl[4], ih[4], il[4];
#pragma unroll
    for (int q2 = 0; q2 < 4; ++q2) {
      const int q = 2 * q2;
      const T u0 = s_u[8 * k8 + q], u1 = s_u[8 * k8 + q + 1];
      if constexpr (CPLX) {
        const float a0 = trh[q] + trl[q], b0 = tih[q] + til[q];              // t = a + i b
        const float a1 = trh[q + 1] + trl[q + 1], b1 = tih[q + 1] + til[q + 1];
        split2_bf16(a0 * u0.x + b0 * u0.y, a1 * u1.x + b1 * u1.y, rh[q2], rl[q2]);   // conj(t) u
        split2_bf16(a0 * u0.y - b0 * u0.x, a1 * u1.y - b1 * u1.x, ih[q2], il[q2]);
      } else {
        split2_bf16((trh[q] + trl[q]) * u0, (trh[q + 1] + trl[q + 1]) * u1, rh[q2], rl[q2]);
      }
    }
    *reinterpret_cast<uint4*>(sBh + offr) = make_uint4(rh[0], rh[1], rh[2], rh[3]);
    *reinterpret_cast<uint4*>(sBl + offr) = make_uint4(rl[0], rl[1], rl[2], rl[3]);
    if constexpr (CPLX) {
      *reinterpret_cast<uint4*>(sBh + offi) = make_uint4(ih[0], ih[1], ih[2], ih[3]);
      *reinterpret_cast<uint4*>(sBl + offi) = make_uint4(il[0], il[1], il[2], il[3]);
    }
    m += dm;
    k8 += dk;
    if (m >= Mp) { m -= Mp; ++k8; }
  }
  umma::fence_proxy_async_smem();     // generic-proxy stores -> visible to the tensor core
  __syncthreads();
  // the MMAs are issued by the last thread, which has no g_a work below (ns * 4 <= 508 sites x groups)
  if (tid == kThreads - 1 && loaded) {
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
    s_issued = 1;
  }
  // while the tensor core runs: g_a[i] = sum_s sigma_si u_s (sigma read from the A tile) and g_b
  T* out = partial + (int64_t)(CL == 2 ? (chunk >> 1) : chunk) * P;
  for (int base = 0; base < ns * 4; base += kThreads) {       // uniform trip count for the shuffles
    const int it = base + tid;
    const bool act = it < ns * 4;
    const int i = act ? (it >> 2) : 0, grp = it & 3;
    T ga = ScalarTraits<T>::zero();
    for (int k = grp; act && loaded && k < KC; k += 4) {
      const uint16_t sb = *reinterpret_cast<const uint16_t*>(sA + umma::kmajor_offset(i, k, 128));
      ga = addx(ga, scal(bf16_val(sb), s_u[k]));
    }
    if constexpr (CPLX) {
      ga.x += __shfl_xor_sync(0xffffffffu, ga.x, 1);
      ga.y += __shfl_xor_sync(0xffffffffu, ga.y, 1);
      ga.x += __shfl_xor_sync(0xffffffffu, ga.x, 2);
      ga.y += __shfl_xor_sync(0xffffffffu, ga.y, 2);
    } else {
      ga += __shfl_xor_sync(0xffffffffu, ga, 1);
      ga += __shfl_xor_sync(0xffffffffu, ga, 2);
    }
    if (act && grp == 0) {
      if constexpr (CL == 2) s_ga[i] = ga;
      else out[i] = ga;
    }
  }
  __syncthreads();
  if (s_issued && !umma::mbar_wait(&bars[1], 0, kWaitLimit)) record_error(status, QES_ERR_TIMEOUT);
  umma::tc_fence_after();
  const int quarter = warp & 3, cg = warp >> 2;
  const int i = 32 * quarter + lane;                      // site row of the accumulator
  const uint32_t lane_addr = tbase + ((uint32_t)(32 * quarter) << 16);
  // The W block of the partial (ns rows of nh) is contiguous in global memory.  When it fits in
  // the operand buffers (free once the MMAs have completed) it is staged there row by row with a
  // padded stride (16-byte row starts, an odd number of 16-byte units: conflict-free vector
  // stores) and then written out by whole warps along each row, so that every store instruction
  // covers consecutive addresses.
  constexpr int EV = 16 / (int)sizeof(T);                 // elements per 16-byte vector
  int ldm = (nh + EV - 1) / EV * EV;
  if (((ldm / EV) & 1) == 0) ldm += EV;
  const bool staged = (size_t)ns * ldm * sizeof(T) <= (size_t)a_bytes + 2u * b_term;
  T* stage = reinterpret_cast<T*>(smem);
  if (s_issued) {
    for (int c = cg; c < Mp / 16; c += kColGroups) {
      const int c0 = 16 * c;
      float gr[16], gi[16];
      if constexpr (CPLX) umma::tmem_ld16x2(lane_addr + c0, lane_addr + d.im_off + c0, gr, gi);
      else umma::tmem_ld16(lane_addr + c0, gr);
      if (staged && i < ns) {
        T* rows = stage + (size_t)i * ldm;
        if (c0 + 16 <= ldm) {
          float4* dst = reinterpret_cast<float4*>(rows + c0);
          if constexpr (CPLX) {
#pragma unroll
            for (int q = 0; q < 8; ++q) dst[q] = make_float4(gr[2 * q], gi[2 * q], gr[2 * q + 1], gi[2 * q + 1]);
          } else {
#pragma unroll
            for (int q = 0; q < 4; ++q) dst[q] = make_float4(gr[4 * q], gr[4 * q + 1], gr[4 * q + 2], gr[4 * q + 3]);
          }
        } else {
#pragma unroll
          for (int q = 0; q < 16; ++q) {
            const int m = c0 + q;
            if (m < nh) {
              if constexpr (CPLX) rows[m] = make_float2(gr[q], gi[q]);
              else rows[m] = gr[q];
            }
          }
        }
      } else if (CL == 2) {
        if (i == 127) {                                   // row 127 = g_b, staged for the pair sum
#pragma unroll
          for (int q = 0; q < 16; ++q) {
            const int m = c0 + q;
            if (m < nh) {
              if constexpr (CPLX) s_gb[m] = make_float2(gr[q], gi[q]);
              else s_gb[m] = gr[q];
            }
          }
        }
      } else if (i < ns || i == 127) {
        T* rowp = (i == 127) ? out + ns : out + ns + nh + (int64_t)i * nh;   // row 127 = g_b
        // 16-byte stores when the row chunk is aligned and complete, element stores otherwise
        const bool vec = (c0 + 16 <= nh) && ((reinterpret_cast<uintptr_t>(rowp + c0) & 15) == 0);
        if (vec) {
          float4* dst = reinterpret_cast<float4*>(rowp + c0);
          if constexpr (CPLX) {
#pragma unroll
            for (int q = 0; q < 8; ++q) dst[q] = make_float4(gr[2 * q], gi[2 * q], gr[2 * q + 1], gi[2 * q + 1]);
          } else {
#pragma unroll
            for (int q = 0; q < 4; ++q) dst[q] = make_float4(gr[4 * q], gr[4 * q + 1], gr[4 * q + 2], gr[4 * q + 3]);
          }
        } else {
#pragma unroll
          for (int q = 0; q < 16; ++q) {
            const int m = c0 + q;
            if (m < nh) {
              if constexpr (CPLX) rowp[m] = make_float2(gr[q], gi[q]);
              else rowp[m] = gr[q];
            }
          }
        }
      }
    }
  }
  if constexpr (CL == 2) {
    if (!s_issued) {                                      // padding chunk or a timed-out load: adds zero
      for (int e = tid; e < ns * ldm; e += kThreads) stage[e] = ScalarTraits<T>::zero();
      for (int e = tid; e < nh; e += kThreads) s_gb[e] = ScalarTraits<T>::zero();
    }
    namespace cgrp = cooperative_groups;
    cgrp::cluster_group cl = cgrp::this_cluster();
    cl.sync();                                            // both partials staged
    const unsigned rank = cl.block_rank();
    const T* peer = cl.map_shared_rank(stage, rank ^ 1u);
    const T* p0 = rank == 0 ? stage : peer;               // rank 0's partial first: fixed order
    const T* p1 = rank == 0 ? peer : stage;
    const int h = (ns + 1) / 2, rb = rank ? h : 0, re = rank ? ns : h;
    T* dstW = out + ns + nh;
    const bool vec = ((reinterpret_cast<uintptr_t>(dstW) & 15) == 0) && (nh % EV == 0);
    for (int r = rb + warp; r < re; r += kWarps) {
      const T* s0r = p0 + (size_t)r * ldm;
      const T* s1r = p1 + (size_t)r * ldm;
      T* dst = dstW + (int64_t)r * nh;
      if (vec) {
        for (int q = lane; q < nh / EV; q += 32) {
          const float4 a = reinterpret_cast<const float4*>(s0r)[q], b = reinterpret_cast<const float4*>(s1r)[q];
          reinterpret_cast<float4*>(dst)[q] = make_float4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w);
        }
      } else {
        for (int q = lane; q < nh; q += 32) dst[q] = addx(s0r[q], s1r[q]);
      }
    }
    if (rank == 0) {
      const T* pga = cl.map_shared_rank(s_ga, 1u);
      for (int e = tid; e < ns; e += kThreads) out[e] = addx(s_ga[e], pga[e]);
    } else {
      const T* pgb = cl.map_shared_rank(s_gb, 0u);
      for (int e = tid; e < nh; e += kThreads) out[ns + e] = addx(pgb[e], s_gb[e]);
    }
    cl.sync();                                            // the peer has read this CTA's staging
  } else if (staged && s_issued) {
    __syncthreads();
    T* dstW = out + ns + nh;
    const bool vec = ((reinterpret_cast<uintptr_t>(dstW) & 15) == 0) && (nh % EV == 0);
    for (int r = warp; r < ns; r += kWarps) {
      const T* src = stage + (size_t)r * ldm;
      T* dst = dstW + (int64_t)r * nh;
      if (vec) {
        for (int q = lane; q < nh / EV; q += 32)
          reinterpret_cast<float4*>(dst)[q] = reinterpret_cast<const float4*>(src)[q];
      } else {
        for (int q = lane; q < nh; q += 32) dst[q] = src[q];
      }
    }
  }
  umma::tc_fence_before();
  __syncthreads();
  if (warp == 0) umma::tmem_dealloc(tbase, d.tmem_cols);
}

// ================================================================================================
// large problems: operands tiled in M (sites) and N (hidden units)
// ================================================================================================
// sig_cols (big): chunk c = MT*128 site rows x KC samples; rows >= ns are zero except row ns,
// which is all ones (D row ns = sum_s Q_s = g_b)
__global__ void tc_sigma_cols_big_kernel(int ns, int R, int KC, int64_t n_samples, int n_chunks,
                                         const uint32_t* __restrict__ bits, uint16_t* __restrict__ out) {
  const int nw = n_words(ns);
  const int64_t items = (int64_t)n_chunks * R * (KC / 8);
  for (int64_t it = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; it < items; it += (int64_t)gridDim.x * blockDim.x) {
    const int r = (int)(it % R);
    const int k8 = (int)((it / R) % (KC / 8));
    const int64_t c = it / ((int64_t)(KC / 8) * R);
    uint16_t v[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int64_t s = c * KC + 8 * k8 + q;
      v[q] = 0;
      if (s < n_samples) {
        if (r < ns) v[q] = ((bits[s * nw + (r >> 5)] >> (r & 31)) & 1u) ? 0x3F80u : 0xBF80u;
        else if (r == ns) v[q] = 0x3F80u;
      }
    }
    uint8_t* base = reinterpret_cast<uint8_t*>(out) + (size_t)c * R * KC * 2;
    *reinterpret_cast<uint4*>(base + umma::kmajor_offset(r, 8 * k8, R)) = pack8(v);
  }
}

// t_cols (big): tile (chunk c, N chunk q, term) = NR rows x KC samples; row n < NC is Re t of hidden
// unit q*NC + n, row NC + n (complex) its Im t
template <class T>
__global__ void tc_t_cols_big_kernel(TcDims d, int64_t n_samples, const T* __restrict__ tt, uint16_t* __restrict__ out) {
  constexpr bool CPLX = ScalarTraits<T>::is_complex;
  const int nh = d.nh, NC = d.NC, NR = d.NR, KC = d.KC, nnc = d.nnc;
  const size_t term_bytes = (size_t)NR * KC * 2;
  const int64_t items = (int64_t)d.n_chunks * nnc * NR * (KC / 8);
  for (int64_t it = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; it < items; it += (int64_t)gridDim.x * blockDim.x) {
    const int n = (int)(it % NR);
    const int k8 = (int)((it / NR) % (KC / 8));
    const int64_t cq = it / ((int64_t)(KC / 8) * NR);         // c * nnc + q
    const int q = (int)(cq % nnc);
    const int64_t c = cq / nnc;
    const bool im = CPLX && n >= NC;
    const int m = q * NC + (im ? n - NC : n);
    uint16_t h[8], l[8];
#pragma unroll
    for (int e = 0; e < 8; ++e) {
      const int64_t s = c * KC + 8 * k8 + e;
      float x = 0.f;
      if (s < n_samples && m < nh) x = im ? tim(tt, s * nh + m) : tre(tt, s * nh + m);
      split_bf16(x, h[e], l[e]);
    }
    uint8_t* base = reinterpret_cast<uint8_t*>(out) + (size_t)cq * 2 * term_bytes;
    const uint32_t off = umma::kmajor_offset(n, 8 * k8, NR);
    *reinterpret_cast<uint4*>(base + off) = pack8(h);
    *reinterpret_cast<uint4*>(base + term_bytes + off) = pack8(l);
  }
}

// O^H u for large problems.  Grid (N chunk, group of SPC sample chunks).  Each sample chunk is
// bulk-copied (Sigma^T: MT*128 x KC, T^T tile: 2 terms x NR x KC) into one of two shared-memory
// buffers while the tensor core works on the other; Q = conj(t) u is formed in place and MT x
// terms x halves MMAs accumulate D[mt][h] (128 sites x NC units) in TMEM across the group.
template <class T>
__global__ void __launch_bounds__(kThreads) tc_ohu_big_kernel(TcDims d, int64_t n_samples, const float2* __restrict__ w,
                                                              const double2* __restrict__ wsum_part, int wsum_n,
                                                              double scale, const uint16_t* __restrict__ sig_cols,
                                                              const uint16_t* __restrict__ t_cols,
                                                              T* __restrict__ partial, int* __restrict__ status,
                                                              const double* __restrict__ cg_done,
                                                              const float* __restrict__ wts) {
  extern __shared__ __align__(128) uint8_t smem[];
  constexpr bool CPLX = ScalarTraits<T>::is_complex;
  constexpr int H = CPLX ? 2 : 1;
  pdl_trigger();
  pdl_wait();                                             // w and its partial sums: previous kernel
  if (cg_block_done(cg_done)) return;                     // converged CG
  const int ns = d.ns, nh = d.nh, KC = d.KC, MT = d.MT, NC = d.NC, NR = d.NR, nnc = d.nnc;
  const int R = MT * 128;
  const uint32_t a_bytes = (uint32_t)R * KC * 2u, b_term = (uint32_t)NR * KC * 2u;
  const uint32_t buf_bytes = a_bytes + 2u * b_term;
  T* s_u = reinterpret_cast<T*>(smem + 2 * buf_bytes);                // [2][KC]
  uint64_t* bars = reinterpret_cast<uint64_t*>(reinterpret_cast<uint8_t*>(s_u + 2 * KC) +
                                               ((16 - (reinterpret_cast<uintptr_t>(s_u + 2 * KC) & 15)) & 15));
  uint64_t* full = bars;          // [2]
  uint64_t* mdone = bars + 2;     // [2]
  uint32_t* tslot = reinterpret_cast<uint32_t*>(bars + 4);
  __shared__ double2 s_mean;
  __shared__ double2 s_red[kWarps];
  __shared__ int s_fail;

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int q = blockIdx.x;                                   // N chunk
  const int g = blockIdx.y;                                   // group of sample chunks
  const int c_first = g * d.SPC;
  const int n_my = min(d.SPC, d.n_chunks - c_first);
  const int64_t P = (int64_t)ns + nh + (int64_t)ns * nh;
  const int n0 = q * NC;
  if (tid == 0) {
    for (int k = 0; k < 4; ++k) umma::mbar_init(&bars[k], 1);
    umma::fence_mbar_init();
    s_fail = 0;
  }
  {
    double2 t = make_double2(0.0, 0.0);
    if (wsum_part && wsum_n > 0)
      for (int k = tid; k < wsum_n; k += kThreads) { t.x += wsum_part[k].x; t.y += wsum_part[k].y; }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      t.x += __shfl_xor_sync(0xffffffffu, t.x, o);
      t.y += __shfl_xor_sync(0xffffffffu, t.y, o);
    }
    if (lane == 0) s_red[warp] = t;
    __syncthreads();
    if (tid == 0) {
      double2 m = make_double2(0.0, 0.0);
      if (wsum_part && wsum_n > 0) {
        for (int k = 0; k < kWarps; ++k) { m.x += s_red[k].x; m.y += s_red[k].y; }
        m.x /= (double)n_samples;
        m.y /= (double)n_samples;
      } else if (wsum_part) {
        m = wsum_part[0];
      }
      s_mean = m;
    }
  }
  if (warp == 0) {
    umma::tmem_alloc(tslot, d.tmem_cols);
    umma::tmem_relinquish();
  }
  umma::tc_fence_before();
  __syncthreads();
  umma::tc_fence_after();
  const uint32_t tbase = *tslot;
  auto issue_load = [&](int j) {               // thread 0 only
    const int c = c_first + j, b = j & 1;
    uint8_t* sb = smem + b * buf_bytes;
    umma::mbar_arrive_expect_tx(&full[b], buf_bytes);
    umma::bulk_g2s(sb, reinterpret_cast<const uint8_t*>(sig_cols) + (size_t)c * a_bytes, a_bytes, &full[b]);
    umma::bulk_g2s(sb + a_bytes, reinterpret_cast<const uint8_t*>(t_cols) + ((size_t)c * nnc + q) * 2 * b_term,
                   2 * b_term, &full[b]);
  };
  if (tid == 0) {
    issue_load(0);
    if (n_my > 1) issue_load(1);
  }
  const float mr = (float)s_mean.x, mi = (float)s_mean.y, fs = (float)scale;
  T ga = ScalarTraits<T>::zero();               // g_a of site tid (q == 0 CTAs)
  bool ok = true;
  for (int j = 0; j < n_my; ++j) {
    const int b = j & 1;
    const int64_t s0 = (int64_t)(c_first + j) * KC;
    uint8_t* sA = smem + b * buf_bytes;
    uint8_t* sBh = sA + a_bytes;
    uint8_t* sBl = sBh + b_term;
    T* u_b = s_u + b * KC;
    for (int k = tid; k < KC; k += kThreads) {
      const int64_t s = s0 + k;
      T u = ScalarTraits<T>::zero();
      if (s < n_samples) {
        const float2 wv = w[s];
        const float f = wts ? fs * wts[s] : fs;
        if constexpr (CPLX) u = make_float2((wv.x - mr) * f, (wv.y - mi) * f);
        else u = (wv.x - mr) * f;
      }
      u_b[k] = u;
    }
    __syncthreads();
    if (ok && !umma::mbar_wait(&full[b], (j >> 1) & 1, kWaitLimit)) {
      record_error(status, QES_ERR_TIMEOUT);
      ok = false;
      s_fail = 1;
    }
    // Q = conj(t) u in place: item (n, k8) = row n (re) and NC + n (im) for 8 samples
    const int items = NC * (KC / 8);
    for (int it = tid; ok && it < items; it += kThreads) {
      const int n = it % NC, k8 = it / NC;
      const uint32_t offr = umma::kmajor_offset(n, 8 * k8, NR);
      float trh[8], trl[8], tih[8], til[8];
      unpack8(*reinterpret_cast<const uint4*>(sBh + offr), trh);
      unpack8(*reinterpret_cast<const uint4*>(sBl + offr), trl);
      uint32_t offi = 0;
      if constexpr (CPLX) {
        offi = umma::kmajor_offset(NC + n, 8 * k8, NR);
        unpack8(*reinterpret_cast<const uint4*>(sBh + offi), tih);
        unpack8(*reinterpret_cast<const uint4*>(sBl + offi), til);
      }
      uint16_t rh[8], rl[8], ih[8], il[8];
#pragma unroll
      for (int e = 0; e < 8; ++e) {
        const T u = u_b[8 * k8 + e];
        if constexpr (CPLX) {
          const float a = trh[e] + trl[e], bb = tih[e] + til[e];
          const float2 qv = make_float2(a * u.x + bb * u.y, a * u.y - bb * u.x);
          split_bf16(qv.x, rh[e], rl[e]);
          split_bf16(qv.y, ih[e], il[e]);
        } else {
          split_bf16((trh[e] + trl[e]) * u, rh[e], rl[e]);
        }
      }
      *reinterpret_cast<uint4*>(sBh + offr) = pack8(rh);
      *reinterpret_cast<uint4*>(sBl + offr) = pack8(rl);
      if constexpr (CPLX) {
        *reinterpret_cast<uint4*>(sBh + offi) = pack8(ih);
        *reinterpret_cast<uint4*>(sBl + offi) = pack8(il);
      }
    }
    umma::fence_proxy_async_smem();
    __syncthreads();
    ok = ok && !s_fail;
    if (tid == 0 && ok) {
      umma::tc_fence_after();
      const uint32_t idesc = umma::idesc_bf16_f32(128, NC);
      const uint32_t aaddr = umma::smem_u32(sA), bh = umma::smem_u32(sBh), bl = umma::smem_u32(sBl);
      for (int kk = 0; kk < KC / 16; ++kk) {
        for (int mt = 0; mt < MT; ++mt) {
          const uint64_t ad = umma::smem_desc(aaddr + (uint32_t)mt * 2048u + 2u * kk * R * 16u, R * 16u, 128u);
          for (int term = 0; term < 2; ++term) {
            const uint32_t bb = term ? bl : bh;
            for (int h = 0; h < H; ++h) {
              const uint64_t bd =
                  umma::smem_desc(bb + (uint32_t)h * (NC / 8) * 128u + 2u * kk * NR * 16u, NR * 16u, 128u);
              umma::mma_bf16(tbase + (uint32_t)((mt * H + h) * NC), ad, bd, idesc,
                             (j > 0 || kk > 0 || term > 0) ? 1u : 0u);
            }
          }
        }
      }
      umma::mma_commit(&mdone[b]);
    }
    // g_a (first N chunk only): thread i sums sigma_si u_s over the chunk from the A tile
    if (q == 0 && ok && tid < ns)
      for (int k = 0; k < KC; ++k) {
        const uint16_t sb = *reinterpret_cast<const uint16_t*>(sA + umma::kmajor_offset(tid, k, R));
        ga = addx(ga, scal(bf16_val(sb), u_b[k]));
      }
    __syncthreads();
    // refill this buffer with chunk j + 2 once the MMAs reading it have completed
    if (tid == 0 && ok && j + 2 < n_my) {
      if (!umma::mbar_wait(&mdone[b], (j >> 1) & 1, kWaitLimit)) {
        record_error(status, QES_ERR_TIMEOUT);
        s_fail = 1;
      } else {
        issue_load(j + 2);
      }
    }
    __syncthreads();
    ok = ok && !s_fail;
  }
  // wait for the last MMAs (each buffer's final commit)
  if (ok) {
    for (int j = max(0, n_my - 2); j < n_my; ++j)
      if (!umma::mbar_wait(&mdone[j & 1], (j >> 1) & 1, kWaitLimit)) {
        record_error(status, QES_ERR_TIMEOUT);
        ok = false;
      }
  }
  umma::tc_fence_after();
  T* out = partial + (int64_t)g * P;
  if (q == 0 && tid < ns) out[tid] = ga;
  const int quarter = warp & 3, cg = warp >> 2;
  for (int mt = 0; ok && mt < MT; ++mt) {
    const int i = mt * 128 + 32 * quarter + lane;             // site row
    const uint32_t lane_addr = tbase + ((uint32_t)(32 * quarter) << 16);
    for (int c = cg; c < NC / 16; c += kColGroups) {
      const int c0 = 16 * c;
      float gr[16], gi[16];
      umma::tmem_ld16(lane_addr + (uint32_t)(mt * H * NC + c0), gr);
      if constexpr (CPLX) umma::tmem_ld16(lane_addr + (uint32_t)((mt * H + 1) * NC + c0), gi);
      if (i <= ns) {
        T* rowp = (i == ns) ? out + ns : out + ns + nh + (int64_t)i * nh;
        const int mb = n0 + c0;
        const bool vec = (mb + 16 <= nh) && ((reinterpret_cast<uintptr_t>(rowp + mb) & 15) == 0);
        if (vec) {
          float4* dst = reinterpret_cast<float4*>(rowp + mb);
          if constexpr (CPLX) {
#pragma unroll
            for (int e = 0; e < 8; ++e) dst[e] = make_float4(gr[2 * e], gi[2 * e], gr[2 * e + 1], gi[2 * e + 1]);
          } else {
#pragma unroll
            for (int e = 0; e < 4; ++e) dst[e] = make_float4(gr[4 * e], gr[4 * e + 1], gr[4 * e + 2], gr[4 * e + 3]);
          }
        } else {
#pragma unroll
          for (int e = 0; e < 16; ++e) {
            const int m = mb + e;
            if (m < nh) {
              if constexpr (CPLX) rowp[m] = make_float2(gr[e], gi[e]);
              else rowp[m] = gr[e];
            }
          }
        }
      }
    }
  }
  umma::tc_fence_before();
  __syncthreads();
  if (warp == 0) umma::tmem_dealloc(tbase, d.tmem_cols);
}

// ================================================================================================
// sv: the whole tensor-core S v in one cooperative launch (single-M-tile problems)
// ================================================================================================
// CTA b takes the 128-sample tiles b, b + G, b + 2G, ... of the G CTAs, all resident (at most one
// per SM).  Phase 1, per tile: w = O v as in tc_ov_kernel (T and V' streamed through a sv_stages-deep
// pipeline, hi*hi + hi*lo + lo*hi MMAs, the spin signs folded in the epilogue); w -> w_out and the
// tile's weighted sum -> wsum_part.  A bounded grid barrier; then every CTA forms the same weighted
// mean of w from the tile sums, in the same order.  Phase 2, per tile: u = wts (w - mean) scale;
// A = Sigma^T (128 sites x 128 samples, +-1, the ones row 127 yields g_b) is written into shared
// memory from the spin words; B = Q^T with Q = conj(t) u is built from the float32 T in chunks of
// SV_QROWS operand rows (BF16 hi/lo), double-buffered, so that the MMAs of one chunk run while the
// next is built.  The MMAs accumulate in TMEM over all of the CTA's tiles and the CTA writes one
// partial P-vector.  A bounded wait that runs out records QES_ERR_TIMEOUT in *status; launches
// that find *status set return at once (the host reports the error after the solve).
constexpr int SV_QROWS = 128;                              // Q^T operand rows per chunk
constexpr uint32_t SV_SIG_BYTES = 128u * 128u * 2u;        // Sigma^T tile: 128 sites x 128 samples
constexpr uint32_t SV_QTERM = SV_QROWS * 128u * 2u;        // one BF16 term of a Q^T chunk
constexpr uint32_t SV_QBUF = 2u * SV_QTERM;                // hi + lo

// count and gen on separate 128-byte lines; waiters poll gen with volatile loads (a sense-reversal
// barrier: the last arrival resets count and advances gen); every wait is bounded
__device__ __forceinline__ void sv_grid_barrier(unsigned int* count, unsigned int* gen, unsigned int nb,
                                                int* status, BarCfg bc) {
  nb += bc.extra;
  __syncthreads();
  if (threadIdx.x == 0) {
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
        if (++it > bc.limit) {
          record_error(status, QES_ERR_TIMEOUT);
          break;
        }
        __nanosleep(20);
      }
    }
    __threadfence();
  }
  __syncthreads();
}

template <class T, class V>
__global__ void __launch_bounds__(kThreads, 1) tc_sv_kernel(TcDims d, int64_t n_samples, const uint32_t* __restrict__ bits,
                                                            const V* __restrict__ v, const T* __restrict__ tt,
                                                            const uint16_t* __restrict__ t_rows,
                                                            const uint16_t* __restrict__ vp, float2* __restrict__ w_out,
                                                            double2* __restrict__ wsum_part, T* __restrict__ partial,
                                                            int* __restrict__ status, const double* __restrict__ cg_done,
                                                            const float* __restrict__ wts, double scale,
                                                            unsigned int* __restrict__ bar, BarCfg bc) {
  extern __shared__ __align__(128) uint8_t smem[];
  constexpr bool CPLX = ScalarTraits<T>::is_complex;
  constexpr int NQ = CPLX ? SV_QROWS / 2 : SV_QROWS;       // hidden units per Q^T chunk
  const int ns = d.ns, nh = d.nh, KCH = d.KCH, NB = d.NB, Sp = d.Sp, Mp = d.Mp;
  const int nK = d.Kd / KCH, S = d.sv_stages;
  const uint32_t a_term = 128u * KCH * 2u, b_term = (uint32_t)NB * KCH * 2u;
  const uint32_t stage_bytes = 2u * (a_term + b_term);
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + d.sv_region);
  uint64_t* empty = full + S;
  uint64_t* done = empty + S;                              // the O v MMAs of one tile
  uint64_t* qbar = done + 1;                               // [2]: the MMAs that read Q^T buffer b
  uint64_t* fin = qbar + 2;                                // every O^H u MMA of the CTA
  uint32_t* tslot = reinterpret_cast<uint32_t*>(fin + 1);
  const int nsp = (ns + 1) & ~1;
  T* s_va = reinterpret_cast<T*>(tslot + 4);
  T* s_ga = s_va + nsp;                                    // g_a, summed over the CTA's tiles
  T* s_u = s_ga + nsp;                                     // u of the current tile
  uint32_t* s_bits = reinterpret_cast<uint32_t*>(s_u + 128);   // spin words, [word][row]
  __shared__ double2 red[kWarps];
  __shared__ float2 s_part[kColGroups][128];
  __shared__ double2 s_mean;
  __shared__ int s_err;

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int G = gridDim.x;
  const int nw = n_words(ns);
  pdl_trigger();
  if (cg_block_done(cg_done)) return;                      // converged CG: nothing to do
  if (tid == 0) s_err = *reinterpret_cast<volatile int*>(status);
  __syncthreads();
  if (s_err != 0) return;                                  // an earlier wait of this solve gave up
  if (tid == 0) {
    for (int q = 0; q < S; ++q) {
      umma::mbar_init(&full[q], 1);
      umma::mbar_init(&empty[q], 1);
    }
    umma::mbar_init(done, 1);
    umma::mbar_init(&qbar[0], 1);
    umma::mbar_init(&qbar[1], 1);
    umma::mbar_init(fin, 1);
    umma::fence_mbar_init();
  }
  if (warp == 0) {
    umma::tmem_alloc(tslot, d.tmem_cols);
    umma::tmem_relinquish();
  }
  for (int i = tid; i < ns; i += kThreads) {
    if constexpr (CPLX) s_va[i] = make_float2(vre(v, i), vim(v, i));
    else s_va[i] = vre(v, i);
    s_ga[i] = ScalarTraits<T>::zero();
  }
  umma::tc_fence_before();
  __syncthreads();
  umma::tc_fence_after();
  const uint32_t tbase = *tslot;
  const uint8_t* gbv = reinterpret_cast<const uint8_t*>(vp);

  // ---------------------------------------------------------------- phase 1: w = O v per tile
  int j = 0;
  for (int tile = blockIdx.x; tile < d.n_tiles; tile += G, ++j) {
    const uint8_t* ga = reinterpret_cast<const uint8_t*>(t_rows) + (size_t)tile * nK * 2 * a_term;
    const int g0 = j * nK;                                 // pipeline chunks issued before this tile
    const int64_t r0 = (int64_t)tile * 128;
    const int rows = (n_samples - r0 < 128) ? (int)(n_samples - r0) : 128;
    if (warp >= 2) {
      // while the pipeline runs: the tile's spin words (epilogue input)
      const int t2 = tid - 64, n2 = kThreads - 64;
      for (int q = t2; q < 128 * nw; q += n2) {
        const int r = q / nw, wd = q - r * nw;
        s_bits[wd * 128 + r] = (r < rows) ? bits[r0 * nw + q] : 0u;
      }
    } else if (warp == 0 && lane == 0) {
      // producer: stage s is refilled once the MMAs that read it have completed
      for (int c = 0; c < nK; ++c) {
        const int g = g0 + c, s = g % S;
        if (g >= S && !umma::mbar_wait(&empty[s], ((g / S) - 1) & 1, kWaitLimit)) {
          record_error(status, QES_ERR_TIMEOUT);
          break;
        }
        uint8_t* stp = smem + s * stage_bytes;
        umma::mbar_arrive_expect_tx(&full[s], stage_bytes);
        umma::bulk_g2s(stp, ga + (size_t)c * 2 * a_term, 2 * a_term, &full[s]);
        umma::bulk_g2s(stp + 2 * a_term, gbv + (size_t)c * 2 * b_term, 2 * b_term, &full[s]);
      }
    } else if (warp == 1 && lane == 0) {
      // MMA issuer: D (128 x NB) += A_hi B_hi + A_hi B_lo + A_lo B_hi over every 16-wide k-step
      const uint32_t idesc = umma::idesc_bf16_f32(128, (uint32_t)NB);
      for (int c = 0; c < nK; ++c) {
        const int g = g0 + c, s = g % S;
        if (!umma::mbar_wait(&full[s], (g / S) & 1, kWaitLimit)) {
          record_error(status, QES_ERR_TIMEOUT);
          break;
        }
        umma::tc_fence_after();
        const uint32_t sa = umma::smem_u32(smem + s * stage_bytes);
        const uint32_t ahi = sa, alo = sa + a_term, bhi = sa + 2 * a_term, blo = bhi + b_term;
        for (int kk = 0; kk < KCH / 16; ++kk) {
          const uint32_t ko_a = 2u * kk * 128u * 16u, ko_b = 2u * kk * NB * 16u;
          const uint64_t dah = umma::smem_desc(ahi + ko_a, 128u * 16u, 128u);
          const uint64_t dal = umma::smem_desc(alo + ko_a, 128u * 16u, 128u);
          const uint64_t dbh = umma::smem_desc(bhi + ko_b, NB * 16u, 128u);
          const uint64_t dbl = umma::smem_desc(blo + ko_b, NB * 16u, 128u);
          umma::mma_bf16(tbase, dah, dbh, idesc, (c > 0 || kk > 0) ? 1u : 0u);
          umma::mma_bf16(tbase, dah, dbl, idesc, 1u);
          umma::mma_bf16(tbase, dal, dbh, idesc, 1u);
        }
        umma::mma_commit(&empty[s]);
      }
      umma::mma_commit(done);                              // every MMA of this tile has completed
    }
    __syncthreads();
    if (!umma::mbar_wait(done, j & 1, kWaitLimit)) record_error(status, QES_ERR_TIMEOUT);
    umma::tc_fence_after();
    // epilogue: warp w reads lane quarter w % 4 (sample rows) and column group w / 4
    {
      const int quarter = warp & 3, cg = warp >> 2;
      const int row = 32 * quarter + lane;
      const bool sval = row < rows;
      const uint32_t* wrd = s_bits + row;                  // word w of this row at wrd[128 w]
      float2 acc = make_float2(0.f, 0.f);
      const uint32_t lane_addr = tbase + ((uint32_t)(32 * quarter) << 16);
      int c = cg;
      for (; c + kColGroups < NB / 16; c += 2 * kColGroups) {
        float y0[16], y1[16];
        umma::tmem_ld16x2(lane_addr + 16 * c, lane_addr + 16 * (c + kColGroups), y0, y1);
        ov_fold16<CPLX>(16 * c, y0, ns, Sp, wrd, nw, acc);
        ov_fold16<CPLX>(16 * (c + kColGroups), y1, ns, Sp, wrd, nw, acc);
      }
      if (c < NB / 16) {
        float y[16];
        umma::tmem_ld16(lane_addr + 16 * c, y);
        ov_fold16<CPLX>(16 * c, y, ns, Sp, wrd, nw, acc);
      }
      // + sigma_s . v_a: column group cg takes the sites of spin words cg, cg + 4, ...
      for (int wd = cg; wd < nw; wd += kColGroups) {
        const uint32_t word = wrd[128 * wd];
        const int i1 = (32 * wd + 32 < ns) ? 32 * wd + 32 : ns;
        float sre = 0.f, sim = 0.f;
        for (int i = 32 * wd; i < i1; ++i) {
          const int sgn = (int)((~word >> (i & 31)) & 1u) << 31;
          const T va = s_va[i];
          if constexpr (CPLX) {
            sre += __int_as_float(__float_as_int(va.x) ^ sgn);
            sim += __int_as_float(__float_as_int(va.y) ^ sgn);
          } else {
            sre += __int_as_float(__float_as_int(va) ^ sgn);
          }
        }
        acc.x += sre;
        acc.y += sim;
      }
      s_part[cg][row] = acc;
      umma::tc_fence_before();
      __syncthreads();
      if (cg == 0) {
        float2 wv = s_part[0][row];
#pragma unroll
        for (int g = 1; g < kColGroups; ++g) wv = wv + s_part[g][row];
        if (!sval) wv = make_float2(0.f, 0.f);
        if (sval) w_out[r0 + row] = wv;
        const double wt = (wts && sval) ? (double)wts[r0 + row] : 1.0;
        double2 ps = make_double2(wt * wv.x, wt * wv.y);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
          ps.x += __shfl_xor_sync(0xffffffffu, ps.x, o);
          ps.y += __shfl_xor_sync(0xffffffffu, ps.y, o);
        }
        if (lane == 0) red[quarter] = ps;
      }
      __syncthreads();
      if (tid == 0) {
        double2 t = make_double2(0.0, 0.0);
        for (int q = 0; q < 4; ++q) { t.x += red[q].x; t.y += red[q].y; }
        wsum_part[tile] = t;
      }
    }
    umma::tc_fence_before();
    __syncthreads();                                       // TMEM read before the next tile's MMAs
  }

  // ---------------------------------------------------------------- the weighted mean of w
  sv_grid_barrier(bar, bar + 32, (unsigned int)G, status, bc);
  {
    double2 t = make_double2(0.0, 0.0);
    for (int q = tid; q < d.n_tiles; q += kThreads) {
      const double2 x = __ldcg(wsum_part + q);
      t.x += x.x;
      t.y += x.y;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      t.x += __shfl_xor_sync(0xffffffffu, t.x, o);
      t.y += __shfl_xor_sync(0xffffffffu, t.y, o);
    }
    if (lane == 0) red[warp] = t;
    __syncthreads();
    if (tid == 0) {
      double2 m = make_double2(0.0, 0.0);
      for (int q = 0; q < kWarps; ++q) { m.x += red[q].x; m.y += red[q].y; }
      s_mean = make_double2(m.x / (double)n_samples, m.y / (double)n_samples);
    }
    __syncthreads();
  }

  // ---------------------------------------------------------------- phase 2: O^H u per tile
  const float mr = (float)s_mean.x, mi = (float)s_mean.y, fs = (float)scale;
  uint8_t* sA = smem;
  uint8_t* sQ = smem + SV_SIG_BYTES;
  const uint32_t a_addr = umma::smem_u32(sA), q_addr = umma::smem_u32(sQ);
  const int nq = (Mp + NQ - 1) / NQ;
  int gq = 0;                                              // Q^T chunks issued by this CTA
  j = 0;
  for (int tile = blockIdx.x; tile < d.n_tiles; tile += G, ++j) {
    const int64_t r0 = (int64_t)tile * 128;
    const int rows = (n_samples - r0 < 128) ? (int)(n_samples - r0) : 128;
    if (j > 0) {
      // the previous tile's MMAs read Sigma^T: wait for its last chunk (and so for all of them)
      if (tid == 0 && !umma::mbar_wait(&qbar[(gq - 1) & 1], ((gq - 1) >> 1) & 1, kWaitLimit))
        record_error(status, QES_ERR_TIMEOUT);
      __syncthreads();
    }
    for (int q = tid; q < 128 * nw; q += kThreads) {
      const int r = q / nw, wd = q - r * nw;
      s_bits[wd * 128 + r] = (r < rows) ? bits[r0 * nw + q] : 0u;
    }
    for (int k = tid; k < 128; k += kThreads) {
      T u = ScalarTraits<T>::zero();
      if (k < rows) {
        const float2 wv = w_out[r0 + k];
        const float f = wts ? fs * wts[r0 + k] : fs;
        if constexpr (CPLX) u = make_float2((wv.x - mr) * f, (wv.y - mi) * f);
        else u = (wv.x - mr) * f;
      }
      s_u[k] = u;
    }
    __syncthreads();
    // Sigma^T: item (site r, samples 8 k8 .. 8 k8 + 7), consecutive threads -> consecutive 16-byte rows
    for (int it = tid; it < 128 * 16; it += kThreads) {
      const int r = it & 127, k8 = it >> 7;
      uint16_t vv[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const int k = 8 * k8 + q;
        uint16_t x = 0;
        if (k < rows) {
          if (r < ns) x = ((s_bits[(r >> 5) * 128 + k] >> (r & 31)) & 1u) ? 0x3F80u : 0xBF80u;
          else if (r == 127) x = 0x3F80u;                  // ones row: D[127] = sum_s Q_s = g_b
        }
        vv[q] = x;
      }
      *reinterpret_cast<uint4*>(sA + umma::kmajor_offset(r, 8 * k8, 128)) = pack8(vv);
    }
    // g_a[i] += sum_s sigma_si u_s (four threads per site, uniform trip count for the shuffles)
    for (int base = 0; base < ns * 4; base += kThreads) {
      const int it = base + tid;
      const bool act = it < ns * 4;
      const int i = act ? (it >> 2) : 0, grp = it & 3;
      T ga = ScalarTraits<T>::zero();
      for (int k = grp; act && k < rows; k += 4) {
        const float sg = ((s_bits[(i >> 5) * 128 + k] >> (i & 31)) & 1u) ? 1.f : -1.f;
        ga = addx(ga, scal(sg, s_u[k]));
      }
      if constexpr (CPLX) {
        ga.x += __shfl_xor_sync(0xffffffffu, ga.x, 1);
        ga.y += __shfl_xor_sync(0xffffffffu, ga.y, 1);
        ga.x += __shfl_xor_sync(0xffffffffu, ga.x, 2);
        ga.y += __shfl_xor_sync(0xffffffffu, ga.y, 2);
      } else {
        ga += __shfl_xor_sync(0xffffffffu, ga, 1);
        ga += __shfl_xor_sync(0xffffffffu, ga, 2);
      }
      if (act && grp == 0) s_ga[i] = addx(s_ga[i], ga);
    }
    for (int h = 0; h < nq; ++h, ++gq) {
      const int b = gq & 1;
      const int m0 = h * NQ, nqu = (Mp - m0 < NQ) ? Mp - m0 : NQ;
      if (gq >= 2) {                                       // buffer b: the MMAs of chunk gq - 2 are done
        if (tid == 0 && !umma::mbar_wait(&qbar[b], ((gq - 2) >> 1) & 1, kWaitLimit))
          record_error(status, QES_ERR_TIMEOUT);
        __syncthreads();
      }
      uint8_t* qb = sQ + b * SV_QBUF;
      // item (unit n, samples 8 k8 .. 8 k8 + 7): consecutive threads take consecutive units, so the
      // loads of T (one sample row at a time) are coalesced and the 16-byte stores conflict-free
      for (int it = tid; it < nqu * 16; it += kThreads) {
        const int n = it % nqu, k8 = it / nqu;
        const int m = m0 + n;
        float qr[8], qi[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          const int k = 8 * k8 + q;
          float tr_ = 0.f, ti_ = 0.f;
          if (m < nh && k < rows) {
            const int64_t e = (r0 + k) * (int64_t)nh + m;
            tr_ = tre(tt, e);
            ti_ = tim(tt, e);
          }
          const T u = s_u[k];
          if constexpr (CPLX) {
            qr[q] = tr_ * u.x + ti_ * u.y;                 // conj(t) u
            qi[q] = tr_ * u.y - ti_ * u.x;
          } else {
            qr[q] = tr_ * u;
            qi[q] = 0.f;
          }
        }
        uint32_t rh[4], rl[4];
#pragma unroll
        for (int q2 = 0; q2 < 4; ++q2) split2_bf16(qr[2 * q2], qr[2 * q2 + 1], rh[q2], rl[q2]);
        const uint32_t offr = umma::kmajor_offset(n, 8 * k8, SV_QROWS);
        *reinterpret_cast<uint4*>(qb + offr) = make_uint4(rh[0], rh[1], rh[2], rh[3]);
        *reinterpret_cast<uint4*>(qb + SV_QTERM + offr) = make_uint4(rl[0], rl[1], rl[2], rl[3]);
        if constexpr (CPLX) {
          uint32_t ih[4], il[4];
#pragma unroll
          for (int q2 = 0; q2 < 4; ++q2) split2_bf16(qi[2 * q2], qi[2 * q2 + 1], ih[q2], il[q2]);
          const uint32_t offi = umma::kmajor_offset(NQ + n, 8 * k8, SV_QROWS);
          *reinterpret_cast<uint4*>(qb + offi) = make_uint4(ih[0], ih[1], ih[2], ih[3]);
          *reinterpret_cast<uint4*>(qb + SV_QTERM + offi) = make_uint4(il[0], il[1], il[2], il[3]);
        }
      }
      umma::fence_proxy_async_smem();                     // generic-proxy stores -> tensor core
      __syncthreads();
      if (tid == kThreads - 1) {
        // D_re[:, m0 ..) (+ D_im[:, im_off + m0 ..)) += Sigma^T Q^T_hi + Sigma^T Q^T_lo over K = 128
        umma::tc_fence_after();
        const uint32_t idesc = umma::idesc_bf16_f32(128, (uint32_t)nqu);
        const uint32_t qa = q_addr + (uint32_t)b * SV_QBUF;
        for (int kk = 0; kk < 8; ++kk) {
          const uint64_t ad = umma::smem_desc(a_addr + 2u * kk * 128u * 16u, 128u * 16u, 128u);
          for (int term = 0; term < 2; ++term) {
            for (int half = 0; half < (CPLX ? 2 : 1); ++half) {
              const uint64_t bd = umma::smem_desc(qa + (uint32_t)term * SV_QTERM + (uint32_t)half * (NQ / 8) * 128u +
                                                      2u * kk * SV_QROWS * 16u,
                                                  SV_QROWS * 16u, 128u);
              umma::mma_bf16(tbase + (uint32_t)(half * d.im_off + m0), ad, bd, idesc,
                             (j > 0 || kk > 0 || term > 0) ? 1u : 0u);
            }
          }
        }
        umma::mma_commit(&qbar[b]);
      }
    }
  }
  if (tid == kThreads - 1) umma::mma_commit(fin);          // arrives once every MMA above is done
  __syncthreads();
  if (!umma::mbar_wait(fin, 0, kWaitLimit)) record_error(status, QES_ERR_TIMEOUT);
  umma::tc_fence_after();

  // ---------------------------------------------------------------- the CTA's partial P-vector
  const int64_t P = (int64_t)ns + nh + (int64_t)ns * nh;
  T* out = partial + (int64_t)blockIdx.x * P;
  const int quarter = warp & 3, cg = warp >> 2;
  const int i = 32 * quarter + lane;                       // site row of the accumulator
  const uint32_t lane_addr = tbase + ((uint32_t)(32 * quarter) << 16);
  // the W block is staged row by row (16-byte row starts, an odd number of 16-byte units) in the
  // freed operand buffers and written out by whole warps along each row
  constexpr int EV = 16 / (int)sizeof(T);
  int ldm = (nh + EV - 1) / EV * EV;
  if (((ldm / EV) & 1) == 0) ldm += EV;
  const bool staged = (size_t)ns * ldm * sizeof(T) <= (size_t)d.sv_region;
  T* stage = reinterpret_cast<T*>(smem);
  for (int c = cg; c < Mp / 16; c += kColGroups) {
    const int c0 = 16 * c;
    float gr[16], gi[16];
    if constexpr (CPLX) umma::tmem_ld16x2(lane_addr + c0, lane_addr + d.im_off + c0, gr, gi);
    else umma::tmem_ld16(lane_addr + c0, gr);
    if (staged && i < ns) {
      T* rw = stage + (size_t)i * ldm;
      if (c0 + 16 <= ldm) {
        float4* dst = reinterpret_cast<float4*>(rw + c0);
        if constexpr (CPLX) {
#pragma unroll
          for (int q = 0; q < 8; ++q) dst[q] = make_float4(gr[2 * q], gi[2 * q], gr[2 * q + 1], gi[2 * q + 1]);
        } else {
#pragma unroll
          for (int q = 0; q < 4; ++q) dst[q] = make_float4(gr[4 * q], gr[4 * q + 1], gr[4 * q + 2], gr[4 * q + 3]);
        }
      } else {
#pragma unroll
        for (int q = 0; q < 16; ++q) {
          const int m = c0 + q;
          if (m < nh) {
            if constexpr (CPLX) rw[m] = make_float2(gr[q], gi[q]);
            else rw[m] = gr[q];
          }
        }
      }
    } else if (i < ns || i == 127) {
      T* rowp = (i == 127) ? out + ns : out + ns + nh + (int64_t)i * nh;   // row 127 = g_b
      const bool vec = (c0 + 16 <= nh) && ((reinterpret_cast<uintptr_t>(rowp + c0) & 15) == 0);
      if (vec) {
        float4* dst = reinterpret_cast<float4*>(rowp + c0);
        if constexpr (CPLX) {
#pragma unroll
          for (int q = 0; q < 8; ++q) dst[q] = make_float4(gr[2 * q], gi[2 * q], gr[2 * q + 1], gi[2 * q + 1]);
        } else {
#pragma unroll
          for (int q = 0; q < 4; ++q) dst[q] = make_float4(gr[4 * q], gr[4 * q + 1], gr[4 * q + 2], gr[4 * q + 3]);
        }
      } else {
#pragma unroll
        for (int q = 0; q < 16; ++q) {
          const int m = c0 + q;
          if (m < nh) {
            if constexpr (CPLX) rowp[m] = make_float2(gr[q], gi[q]);
            else rowp[m] = gr[q];
          }
        }
      }
    }
  }
  for (int e = tid; e < ns; e += kThreads) out[e] = s_ga[e];
  if (staged) {
    __syncthreads();
    T* dstW = out + ns + nh;
    const bool vec = ((reinterpret_cast<uintptr_t>(dstW) & 15) == 0) && (nh % EV == 0);
    for (int r = warp; r < ns; r += kWarps) {
      const T* src = stage + (size_t)r * ldm;
      T* dst = dstW + (int64_t)r * nh;
      if (vec) {
        for (int q = lane; q < nh / EV; q += 32)
          reinterpret_cast<float4*>(dst)[q] = reinterpret_cast<const float4*>(src)[q];
      } else {
        for (int q = lane; q < nh; q += 32) dst[q] = src[q];
      }
    }
  }
  umma::tc_fence_before();
  __syncthreads();
  if (warp == 0) umma::tmem_dealloc(tbase, d.tmem_cols);
}

// ================================================================================================
// host side
// ================================================================================================
static int pow2_at_least(int x) {
  int p = 32;
  while (p < x) p <<= 1;
  return p;
}

// tiling overrides (qes_sr_set_tiling): 0 = automatic, 1 = single-M-tile kernel, 2 = M/N-tiled kernel;
// hidden units per N chunk and target CTA count of the M/N-tiled O^H u (0 = automatic)
static std::atomic<int> g_tile_mode{0}, g_tile_nc{0}, g_tile_ctas{0};
// split-complex O v (V'' operand) where NB <= 256: off by default (heis10x10 CG iteration 45.0 us with
// it, 44.9 us without: O v is bound by its MMAs, not by the direction operand it halves)
static std::atomic<int> g_ov_split{0};
extern "C" int qes_sr_set_ov_split(int on) {
  g_ov_split.store(on ? 1 : 0);
  return QES_OK;
}
// O v through z = Sigma V (tc_ovz_kernel) where its operands fit: on by default
static std::atomic<int> g_ovz{1};
// L2 prefetch of tc_ovz_kernel's T tile before it waits on its predecessor: off by default
// (heis10x10 CG iteration 42.3 us with it, 42.1 us without; 6x6 J1-J2 28.8 both: T already stays
// in L2 between iterations)
static std::atomic<int> g_prefetch{0};
extern "C" int qes_sr_set_prefetch(int on) {
  g_prefetch.store(on ? 1 : 0);
  return QES_OK;
}
extern "C" int qes_sr_set_ovz(int on) {
  g_ovz.store(on ? 1 : 0);
  return QES_OK;
}
static std::atomic<int> g_ohu_pairs{0};      // measured slower on B200 (heis 10x10: 49.5 vs 46.2 us per CG iteration)
// fused S v kernel where the tiling admits it: off by default (heis10x10 CG iteration 54.6 us with it,
// 44.2 us with the O v / O^H u pair: its per-tile phases run one after another behind block barriers)
static std::atomic<int> g_sv{0};
extern "C" int qes_sr_set_ohu_pairs(int on) {
  g_ohu_pairs.store(on ? 1 : 0);
  return QES_OK;
}
extern "C" int qes_sr_set_fused_sv(int on) {
  g_sv.store(on ? 1 : 0);
  return QES_OK;
}

// SM count of the current device (cached per device; 148 when it cannot be read)
static int tc_sm_count() {
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
extern "C" int qes_sr_set_tiling(int mode, int nc, int ctas) {
  if (mode < 0 || mode > 2 || nc < 0 || (nc % 16) != 0 || ctas < 0) {
    qes_set_last_message("qes_sr_set_tiling: mode 0..2, nc a multiple of 16 (or 0), ctas >= 0");
    return QES_ERR_ARG;
  }
  g_tile_mode.store(mode);
  g_tile_nc.store(nc);
  g_tile_ctas.store(ctas);
  return QES_OK;
}

bool tc_plan(int dtype, int ns, int nh, int64_t n_samples, TcDims* dout) {
  const bool cplx = dtype == QES_DTYPE_C64;
  const int H = cplx ? 2 : 1;
  TcDims t{};
  t.ns = ns;
  t.nh = nh;
  t.Mp = (nh + 15) / 16 * 16;
  t.Np = cplx ? 2 * t.Mp : t.Mp;
  t.Sp = cplx ? (ns + 1 + 7) / 8 * 8 : (ns + 1 + 15) / 16 * 16;  // sites + the v_b row
  t.NB = cplx ? 2 * t.Sp : t.Sp;
  // complex O v as two products against V'' (two accumulators of NB <= 256 columns), K chunks of 16
  // so that the Re t and Im t chunks of the same hidden units pair up
  t.splitc = cplx && t.NB <= 256 && g_ov_split.load() != 0;
  t.KCH = t.splitc ? 16 : 32;
  t.Kd = cplx ? 2 * t.Mp : (nh + 31) / 32 * 32;               // multiple of KCH
  t.VK = t.splitc ? t.Mp : t.Kd;
  if (n_samples < 1 || t.Kd % t.KCH != 0 || t.VK % t.KCH != 0 || t.NB > 512) return false;
  const size_t tsz = cplx ? 8 : 4;
  // ov: as many pipeline stages (2..4, 2..6 split) as shared memory holds
  const size_t a_term = 128u * t.KCH * 2, b_term = (size_t)t.NB * t.KCH * 2;
  const size_t stage = t.splitc ? 4u * a_term + 2u * b_term : 2u * (a_term + b_term);
  const int smax = t.splitc ? 6 : 4;
  const size_t ov_extra = 8 * (2 * smax + 1) + 16 + ((size_t)ns * tsz + 15) / 16 * 16 + 128u * 4u * ((ns + 31) / 32) + 64;
  const int S = (int)std::min<size_t>(smax, (kTcSmemLimit - ov_extra) / stage);
  if (S < 2) return false;
  t.ov_stages = S;
  t.ov_smem = (int)(S * stage + ov_extra);
  // ovz operands: A (128 x Kz) and the whole Bz (NZ x Kz, hi/lo) in shared memory, NZ TMEM columns
  t.Kz = (ns + 1 + 15) / 16 * 16;
  t.NZ = cplx ? 2 * t.Mp : t.Mp;
  {
    const size_t zsm = 128u * t.Kz * 2 + (size_t)t.Kz * t.NZ * 4 + 8u * (t.Kz / 16 + 1) + 16 +
                       ((size_t)ns * tsz + 15) / 16 * 16 + 128u * 4u * ((ns + 31) / 32) + 64;
    // an explicit request for the split-complex product or the fused S v kernel (both read V') wins
    t.ovz = g_ovz.load() != 0 && !t.splitc && g_sv.load() == 0 && t.NZ <= 512 && zsm <= kTcSmemLimit;
    t.ovz_smem = (int)zsm;
    t.ovz_tmem = pow2_at_least(std::max(t.NZ, 32));
    t.prefetch = g_prefetch.load() != 0;
  }
  t.n_tiles = (int)((n_samples + 127) / 128);
  t.big = ns > 127 || t.Mp > 256 || t.NB > 256;
  const int mode = g_tile_mode.load();
  if (mode == 2) t.big = true;
  if (mode == 1 && t.big) return false;
  if (!t.big) {
    t.im_off = pow2_at_least(t.Mp);
    t.tmem_cols = pow2_at_least(std::max(cplx ? 2 * t.im_off : t.im_off, t.splitc ? 256 + t.NB : t.NB));
    if (t.tmem_cols > 512) return false;
    int kc = 256;
    while (kc >= 16) {
      const size_t sm = 128u * kc * 2 + 2u * t.Np * kc * 2 + (size_t)(kc + nh + ns) * tsz + 64;
      if (sm <= kTcSmemLimit) break;
      kc -= 16;
    }
    if (kc < 16) return false;
    t.KC = kc;
    t.n_chunks = (int)((n_samples + kc - 1) / kc);
    // pairs of O^H u CTAs (thread-block clusters of two) when the W block of a partial fits the
    // operand buffers (the kernel's staging stride: 16-byte rows, an odd number of 16-byte units)
    const int ev = (int)(16 / tsz);
    int ldm = (nh + ev - 1) / ev * ev;
    if (((ldm / ev) & 1) == 0) ldm += ev;
    const bool fits = (size_t)ns * ldm * tsz <= 128u * kc * 2 + 2u * t.Np * kc * 2;
    t.cl = (g_ohu_pairs.load() && fits && t.n_chunks >= 2) ? 2 : 1;
    t.nsplit = (t.n_chunks + t.cl - 1) / t.cl;
    t.ohu_smem = (int)(128u * kc * 2 + 2u * t.Np * kc * 2 + (size_t)(kc + nh + ns) * tsz + 64);
    // fused S v: the shared region holds the O v pipeline, later Sigma^T and two Q^T buffers; one CTA
    // per SM at most (launch bounds cap the registers at 128 per thread), so sv_grid CTAs are resident
    if (g_sv.load() != 0 && !t.splitc && !t.ovz) {          // the fused kernel reads the [Re | -Im ; Im | Re] V'
      const int nsp = (ns + 1) & ~1, nw = (ns + 31) / 32;
      for (int S2 = 4; S2 >= 2 && !t.sv; --S2) {
        const size_t region = std::max<size_t>((size_t)S2 * stage, SV_SIG_BYTES + 2u * SV_QBUF);
        const size_t extra = 8u * (2 * S2 + 4) + 16 + (size_t)(2 * nsp + 128) * tsz + 512u * nw + 16;
        if (region + extra <= kTcSmemLimit) {
          t.sv = true;
          t.sv_stages = S2;
          t.sv_region = (int)region;
          t.sv_smem = (int)(region + extra);
        }
      }
      t.sv_grid = (int)std::min<int64_t>(t.n_tiles, tc_sm_count());
    }
    *dout = t;
    return true;
  }
  // large problems: O^H u tiled in M (sites + ones row) and N (hidden units)
  t.MT = (ns + 1 + 127) / 128;
  if (t.MT > 4) return false;                                  // TMEM: MT * H * NC <= 512 with NC >= 16
  int nc = (512 / (t.MT * H)) / 16 * 16;
  nc = std::min(nc, 256);
  nc = std::min(nc, t.Mp);
  if (g_tile_nc.load() > 0) nc = std::min(nc, g_tile_nc.load());
  if (nc < 16) return false;
  t.NC = nc;
  t.NR = H * nc;
  t.nnc = (nh + nc - 1) / nc;
  const size_t R = (size_t)t.MT * 128;
  int kc = 256;
  while (kc >= 16) {
    const size_t sm = 2u * (R * kc * 2 + 2u * t.NR * kc * 2) + 2u * kc * tsz + 16 + 8 * 4 + 16 + 64;
    if (sm <= kTcSmemLimit) break;
    kc -= 16;
  }
  if (kc < 16) return false;
  t.KC = kc;
  t.n_chunks = (int)((n_samples + kc - 1) / kc);
  const int ctas = g_tile_ctas.load() > 0 ? g_tile_ctas.load() : 2 * 148;
  const int groups_target = std::max(1, (ctas + t.nnc - 1) / t.nnc);
  t.SPC = std::max(1, (t.n_chunks + groups_target - 1) / groups_target);
  t.nsplit = (t.n_chunks + t.SPC - 1) / t.SPC;
  t.ohu_smem = (int)(2u * (R * kc * 2 + 2u * t.NR * kc * 2) + 2u * kc * tsz + 16 + 8 * 4 + 16 + 64);
  t.im_off = 0;
  t.cl = 1;
  t.tmem_cols = pow2_at_least(std::max(t.MT * H * t.NC, t.splitc ? 256 + t.NB : t.NB));
  if (t.tmem_cols > 512) return false;
  *dout = t;
  return true;
}

static size_t al256(size_t x) { return (x + 255) & ~(size_t)255; }
static size_t sz_t_rows(const TcDims& d) { return (size_t)d.n_tiles * 128 * d.Kd * 2 * 2; }
static size_t sz_t_cols(const TcDims& d) {
  return d.big ? (size_t)d.n_chunks * d.nnc * d.NR * d.KC * 2 * 2 : (size_t)d.n_chunks * d.Np * d.KC * 2 * 2;
}
static size_t sz_sig_cols(const TcDims& d) { return (size_t)d.n_chunks * (d.big ? d.MT * 128 : 128) * d.KC * 2; }
// the direction-vector operand buffer holds V' or Bz (sized for both, so that switching forms
// between calls needs no new workspace)
static size_t sz_vp(const TcDims& d) { return std::max((size_t)d.NB * d.VK * 2 * 2, (size_t)d.Kz * d.NZ * 4); }

size_t tc_workspace_bytes(const TcDims& d) {
  return al256(sz_t_rows(d)) + al256(sz_t_cols(d)) + al256(sz_sig_cols(d)) + al256(sz_vp(d)) +
         al256((size_t)d.n_tiles * sizeof(double2)) + al256(sizeof(int) * 4) + al256(sizeof(unsigned int) * 64);
}

TcWork tc_layout(const TcDims& d, char* base) {
  TcWork w{};
  size_t off = 0;
  w.t_rows = (uint16_t*)(base + off); off += al256(sz_t_rows(d));
  w.t_cols = (uint16_t*)(base + off); off += al256(sz_t_cols(d));
  w.sig_cols = (uint16_t*)(base + off); off += al256(sz_sig_cols(d));
  w.vp = (uint16_t*)(base + off); off += al256(sz_vp(d));
  w.wsum = (double2*)(base + off); off += al256((size_t)d.n_tiles * sizeof(double2));
  w.status = (int*)(base + off); off += al256(sizeof(int) * 4);
  w.bar = (unsigned int*)(base + off); off += al256(sizeof(unsigned int) * 64);
  return w;
}

template <class T, class V>
static int tc_set_attrs() {
  QES_CUDA_CHECK(cudaFuncSetAttribute(tc_ov_kernel<T, V>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)kTcSmemLimit));
  QES_CUDA_CHECK(cudaFuncSetAttribute(tc_ohu_kernel<T, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)kTcSmemLimit));
  QES_CUDA_CHECK(cudaFuncSetAttribute(tc_ohu_kernel<T, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)kTcSmemLimit));
  QES_CUDA_CHECK(cudaFuncSetAttribute(tc_ohu_big_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)kTcSmemLimit));
  QES_CUDA_CHECK(cudaFuncSetAttribute(tc_sv_kernel<T, V>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)kTcSmemLimit));
  QES_CUDA_CHECK(cudaFuncSetAttribute(tc_ovz_kernel<T, V>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)kTcSmemLimit));
  return QES_OK;
}

// O^H u of the single-M-tile path: one CTA per sample chunk, or clusters of two CTAs (d.cl == 2, the
// grid padded to an even size) that add their partials on chip; chained to the previous kernel by PDL
template <class T>
static int launch_tc_ohu(const TcDims& d, int64_t n_samples, const float2* g, const double2* gsum_part, int gsum_n,
                         double scale, const TcWork& w, T* partial, cudaStream_t st,
                         const double* cg_done = nullptr) {
  if (d.cl == 2) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)((d.n_chunks + 1) & ~1));
    cfg.blockDim = dim3(kThreads);
    cfg.dynamicSmemBytes = (size_t)d.ohu_smem;
    cfg.stream = st;
    cudaLaunchAttribute at[2];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = 2;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    at[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[1].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = qes_pdl_on() ? 2 : 1;
    QES_CUDA_CHECK(cudaLaunchKernelEx(&cfg, tc_ohu_kernel<T, 2>, d, n_samples, g, gsum_part, gsum_n, scale,
                                      (const uint16_t*)w.sig_cols, (const uint16_t*)w.t_cols, partial, w.status,
                                      cg_done, w.wts));
  } else {
    QES_CUDA_CHECK(qes_launch_pdl(tc_ohu_kernel<T, 1>, dim3(d.n_chunks), dim3(kThreads), (size_t)d.ohu_smem, st, d,
                                  n_samples, g, gsum_part, gsum_n, scale, (const uint16_t*)w.sig_cols,
                                  (const uint16_t*)w.t_cols, partial, w.status, cg_done, w.wts));
  }
  return QES_OK;
}

int tc_prepare_step(int dtype, const TcDims& d, int64_t n_samples, const uint32_t* bits, const void* tanh_theta,
                    const TcWork& w, cudaStream_t st) {
  int rc = (dtype == QES_DTYPE_C64) ? tc_set_attrs<float2, double2>() : tc_set_attrs<float, double>();
  if (rc) return rc;
  QES_CUDA_CHECK(cudaMemsetAsync(w.status, 0, sizeof(int), st));
  QES_CUDA_CHECK(cudaMemsetAsync(w.bar, 0, sizeof(unsigned int) * 64, st));
  if (d.big)
    tc_sigma_cols_big_kernel<<<1184, 256, 0, st>>>(d.ns, d.MT * 128, d.KC, n_samples, d.n_chunks, bits, w.sig_cols);
  else
    tc_sigma_cols_kernel<<<1184, 256, 0, st>>>(d.ns, d.KC, n_samples, d.n_chunks, bits, w.sig_cols);
  QES_LAUNCH_CHECK();
  // tc_ovz_kernel reads T transposed per tile (in the t_rows buffer, which holds it: 128 x 2 Mp x 4
  // bytes per tile >= 128 x nh x 8 complex, 128 x Kd x 4 >= 128 x nh x 4 real)
  const bool rows = !d.ovz || d.sv;
  if (!rows) {
    const int64_t squares = (int64_t)d.n_tiles * 4 * ((d.nh + 31) / 32);
    const int grid = (int)std::min<int64_t>(squares, 4096);
    if (dtype == QES_DTYPE_C64)
      tc_t_tiles_kernel<float2><<<grid, dim3(32, 8), 0, st>>>(d.nh, n_samples, d.n_tiles, (const float2*)tanh_theta,
                                                              reinterpret_cast<float2*>(w.t_rows));
    else
      tc_t_tiles_kernel<float><<<grid, dim3(32, 8), 0, st>>>(d.nh, n_samples, d.n_tiles, (const float*)tanh_theta,
                                                             reinterpret_cast<float*>(w.t_rows));
    QES_LAUNCH_CHECK();
  }
  if (dtype == QES_DTYPE_C64) {
    if (rows) tc_t_rows_kernel<float2><<<1184, 256, 0, st>>>(d, n_samples, (const float2*)tanh_theta, w.t_rows);
    if (d.big) tc_t_cols_big_kernel<float2><<<1184, 256, 0, st>>>(d, n_samples, (const float2*)tanh_theta, w.t_cols);
    else tc_t_cols_kernel<float2><<<1184, 256, 0, st>>>(d, n_samples, (const float2*)tanh_theta, w.t_cols);
    QES_LAUNCH_CHECK_N(2);
  } else {
    if (rows) tc_t_rows_kernel<float><<<1184, 256, 0, st>>>(d, n_samples, (const float*)tanh_theta, w.t_rows);
    if (d.big) tc_t_cols_big_kernel<float><<<1184, 256, 0, st>>>(d, n_samples, (const float*)tanh_theta, w.t_cols);
    else tc_t_cols_kernel<float><<<1184, 256, 0, st>>>(d, n_samples, (const float*)tanh_theta, w.t_cols);
    QES_LAUNCH_CHECK_N(2);
  }
  return QES_OK;
}

// the direction-vector operand of the O v kernel in use (V' or Bz), built from v
template <class V>
static int tc_build_operand(const TcDims& d, bool cplx, const V* v, const TcWork& w, cudaStream_t st) {
  if (d.ovz) {
    const int items = d.NZ * (d.Kz / 8);
    tc_build_vz_kernel<V><<<(items + 255) / 256, 256, 0, st>>>(d, cplx, v, w.vp);
  } else {
    const int items = d.NB * (d.VK / 8);
    tc_build_vp_kernel<V><<<(items + 255) / 256, 256, 0, st>>>(d, cplx, v, w.vp);
  }
  QES_LAUNCH_CHECK();
  return QES_OK;
}

template <class T, class V>
static int tc_matvec_t(const TcDims& d, int64_t n_samples, const uint32_t* bits, const T* tt, const V* v,
                       float2* w_out, T* partial, const TcWork& w, cudaStream_t st, bool build_vp,
                       const double* cg_done, BarCfg bc) {
  const bool cplx = ScalarTraits<T>::is_complex;
  if (d.sv) {
    // one cooperative launch (every CTA resident: the mean of w is a grid barrier), after an
    // ordinary launch that builds V' on the first iteration
    if (build_vp) {
      const int items = d.NB * (d.VK / 8);
      tc_build_vp_kernel<V><<<(items + 255) / 256, 256, 0, st>>>(d, cplx, v, w.vp);
      QES_LAUNCH_CHECK();
    }
    const int pf = qes_prof_begin(QES_PROF_SV, st);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)d.sv_grid);
    cfg.blockDim = dim3(kThreads);
    cfg.dynamicSmemBytes = (size_t)d.sv_smem;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeCooperative;
    at[0].val.cooperative = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    QES_CUDA_CHECK(cudaLaunchKernelEx(&cfg, tc_sv_kernel<T, V>, d, n_samples, bits, v, tt,
                                      (const uint16_t*)w.t_rows, (const uint16_t*)w.vp, w_out, w.wsum, partial,
                                      w.status, cg_done, w.wts, 1.0 / (double)n_samples, w.bar, bc));
    QES_LAUNCH_CHECK();
    qes_prof_end(pf, st);
    return QES_OK;
  }
  // the CG iteration's kernels form a programmatic-dependent-launch chain (qes_launch_pdl)
  if (build_vp) {
    // first iteration: an ordinary launch, so that everything before it (the setup that clears the
    // converged flag of the previous solve) has completed before the PDL chain begins; the flag is
    // read by tc_ov / tc_ohu before they wait on their predecessor
    if (int rc = tc_build_operand<V>(d, cplx, v, w, st)) return rc;
  }
  int pf = qes_prof_begin(QES_PROF_OV, st);
  if (d.ovz)
    QES_CUDA_CHECK(qes_launch_pdl(tc_ovz_kernel<T, V>, dim3(d.n_tiles), dim3(kThreads), (size_t)d.ovz_smem, st, d,
                                  n_samples, bits, v, reinterpret_cast<const T*>(w.t_rows), (const uint16_t*)w.vp,
                                  w_out, w.wsum, w.status, cg_done, w.wts));
  else
    QES_CUDA_CHECK(qes_launch_pdl(tc_ov_kernel<T, V>, dim3(d.n_tiles), dim3(kThreads), (size_t)d.ov_smem, st, d,
                                  n_samples, bits, v, (const uint16_t*)w.t_rows, (const uint16_t*)w.vp, w_out, w.wsum,
                                  w.status, cg_done, w.wts));
  QES_LAUNCH_CHECK();
  qes_prof_end(pf, st);
  pf = qes_prof_begin(QES_PROF_OHU, st);
  const double inv_n = 1.0 / (double)n_samples;
  if (d.big)
    QES_CUDA_CHECK(qes_launch_pdl(tc_ohu_big_kernel<T>, dim3(d.nnc, d.nsplit), dim3(kThreads), (size_t)d.ohu_smem, st,
                                  d, n_samples, (const float2*)w_out, (const double2*)w.wsum, d.n_tiles, inv_n,
                                  (const uint16_t*)w.sig_cols, (const uint16_t*)w.t_cols, partial, w.status,
                                  cg_done, w.wts));
  else if (int rc = launch_tc_ohu<T>(d, n_samples, w_out, w.wsum, d.n_tiles, inv_n, w, partial, st, cg_done))
    return rc;
  QES_LAUNCH_CHECK();
  qes_prof_end(pf, st);
  return QES_OK;
}

template <class T, class V>
static int tc_ov_t(const TcDims& d, int64_t n_samples, const uint32_t* bits, const T* tt, const V* v, float2* w_out,
                   const TcWork& w, cudaStream_t st) {
  const bool cplx = ScalarTraits<T>::is_complex;
  if (int rc = tc_build_operand<V>(d, cplx, v, w, st)) return rc;
  const int pf = qes_prof_begin(QES_PROF_OV, st);
  if (d.ovz)
    tc_ovz_kernel<T, V><<<d.n_tiles, kThreads, d.ovz_smem, st>>>(d, n_samples, bits, v,
                                                               reinterpret_cast<const T*>(w.t_rows), w.vp, w_out,
                                                               w.wsum, w.status, nullptr, w.wts);
  else
    tc_ov_kernel<T, V><<<d.n_tiles, kThreads, d.ov_smem, st>>>(d, n_samples, bits, v, w.t_rows, w.vp, w_out, w.wsum,
                                                             w.status, nullptr, w.wts);
  QES_LAUNCH_CHECK();
  qes_prof_end(pf, st);
  return QES_OK;
}

int tc_ov(int dtype, const TcDims& d, int64_t n_samples, const uint32_t* bits, const void* tanh_theta, const void* v,
          float2* w_out, const TcWork& w, cudaStream_t st) {
  if (dtype == QES_DTYPE_C64)
    return tc_ov_t<float2, double2>(d, n_samples, bits, (const float2*)tanh_theta, (const double2*)v, w_out, w, st);
  return tc_ov_t<float, double>(d, n_samples, bits, (const float*)tanh_theta, (const double*)v, w_out, w, st);
}

int tc_matvec(int dtype, const TcDims& d, int64_t n_samples, const uint32_t* bits, const void* tanh_theta,
              const void* v, float2* w_out, void* partial, const TcWork& w, cudaStream_t st, bool build_vp,
              const double* cg_done, BarCfg bc) {
  if (dtype == QES_DTYPE_C64)
    return tc_matvec_t<float2, double2>(d, n_samples, bits, (const float2*)tanh_theta, (const double2*)v, w_out,
                                        (float2*)partial, w, st, build_vp, cg_done, bc);
  return tc_matvec_t<float, double>(d, n_samples, bits, (const float*)tanh_theta, (const double*)v, w_out,
                                    (float*)partial, w, st, build_vp, cg_done, bc);
}

int tc_ohu(int dtype, const TcDims& d, int64_t n_samples, const float2* g, const double2* gsum_part, int gsum_n,
           double scale, void* partial, const TcWork& w, cudaStream_t st) {
  if (d.big) {
    if (dtype == QES_DTYPE_C64)
      tc_ohu_big_kernel<float2><<<dim3(d.nnc, d.nsplit), kThreads, d.ohu_smem, st>>>(
          d, n_samples, g, gsum_part, gsum_n, scale, w.sig_cols, w.t_cols, (float2*)partial, w.status, nullptr, w.wts);
    else
      tc_ohu_big_kernel<float><<<dim3(d.nnc, d.nsplit), kThreads, d.ohu_smem, st>>>(
          d, n_samples, g, gsum_part, gsum_n, scale, w.sig_cols, w.t_cols, (float*)partial, w.status, nullptr, w.wts);
  } else if (dtype == QES_DTYPE_C64) {
    if (int rc = launch_tc_ohu<float2>(d, n_samples, g, gsum_part, gsum_n, scale, w, (float2*)partial, st)) return rc;
  } else {
    if (int rc = launch_tc_ohu<float>(d, n_samples, g, gsum_part, gsum_n, scale, w, (float*)partial, st)) return rc;
  }
  QES_LAUNCH_CHECK();
  return QES_OK;
}
