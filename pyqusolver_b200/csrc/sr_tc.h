// Internal interface of the tensor-core SR matvec (sr_tc.cu) used by sr.cu.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

struct TcDims {
  int ns, nh;        // sites, hidden units
  int Mp;            // hidden units padded to 16 (N of one ohu MMA)
  int Np;            // ohu B rows: 2*Mp (complex) or Mp (real)
  int Kd;            // ov K: 2*Mp (complex: [Re t | Im t]) or nh padded to KCH (real)
  int KCH;           // ov K chunk per pipeline stage
  // complex O v with NB <= 256 (splitc): two products T_re V''^T and T_im V''^T into two TMEM
  // accumulators (columns 0 and 256), V'' = [Re v rows ; Im v rows] over K = the hidden units (VK =
  // Mp): half the bytes of the [Re | -Im ; Im | Re] operand that every O v CTA reads; otherwise VK = Kd
  bool splitc;
  int VK;
  int Sp;            // sites + the v_b row, padded (rows of one Y half)
  int NB;            // ov N: 2*Sp (complex) or Sp (real)
  int KC;            // samples per ohu chunk (K of the ohu GEMM, multiple of 16)
  int im_off;        // TMEM column offset of the imaginary half (ohu)
  int tmem_cols;     // TMEM columns allocated per CTA
  int n_tiles;       // ceil(Ns / 128)
  int n_chunks;      // ceil(Ns / KC)
  int ov_smem, ohu_smem;
  int ov_stages;     // ov pipeline depth (2..4, as many as fit shared memory)
  int nsplit;        // partial P-vectors written by one O^H u pass
  int cl;            // O^H u CTAs per thread-block cluster (2: pairs sum their partials on chip)
  // large problems (ns > 127 or more hidden units than one MMA N): the O^H u GEMM is tiled in
  // M (MT tiles of 128 sites, the ones row at site index ns) and N (nnc chunks of NC hidden units,
  // NR = NC (real) or 2 NC (complex) operand rows), and one CTA folds SPC sample chunks into TMEM
  bool big;
  int MT, NC, NR, nnc, SPC;
  // fused S v (tc_sv_kernel, single-M-tile problems): one cooperative launch of sv_grid CTAs, each
  // taking every sv_grid-th 128-sample tile and writing one partial P-vector; sv_region bytes of
  // shared memory hold the O v pipeline (sv_stages stages), then Sigma^T and two Q^T chunk buffers
  bool sv;
  int sv_grid, sv_stages, sv_region, sv_smem;
  // O v through z = Sigma V (tc_ovz_kernel): A = the spins and a ones column (128 samples x Kz,
  // Kz = sites + 1 padded to 16, exact in BF16), B = Bz (NZ rows x Kz, hi/lo): row m is Re V_{.,m},
  // row Mp + m (complex) is Im V_{.,m}, K index ns holds v_b; (O v)_s = sum_m t_sm z_sm + sigma_s . v_a
  // with t in float32.  Bz replaces V' in the direction-vector buffer when ovz is set.
  bool ovz;
  int Kz, NZ, ovz_smem, ovz_tmem;
  bool prefetch;     // tc_ovz_kernel pulls its T tile into L2 before waiting on its predecessor
};

// Configuration of a bounded grid barrier: `extra` arrivals that never come and a short poll limit
// make every wait run out (a test hook); zero / kGridBarLimit in normal use.
struct BarCfg { unsigned int extra; unsigned int limit; };
constexpr unsigned int kGridBarLimit = 1u << 24;     // polls (with a short sleep) before giving up

struct TcWork {
  uint16_t* t_rows;     // ov A: per tile and K chunk, hi/lo BF16 tiles of T
  uint16_t* t_cols;     // ohu B before scaling: per sample chunk, hi/lo BF16 tiles of T^T
  uint16_t* sig_cols;   // ohu A: per sample chunk, Sigma^T (128 x KC) BF16
  uint16_t* vp;         // ov B: V' hi/lo BF16 tiles (per CG iteration)
  double2* wsum;        // n_tiles partial sums of w = O v (weighted by wts when given)
  int* status;          // first error code of a bounded wait
  unsigned int* bar;    // grid barrier of tc_sv_kernel: count at [0], generation at [32]
  const float* wts;     // per-sample weights normalised to sum Ns (nullptr: uniform); set per call
};

constexpr size_t kTcSmemLimit = 220 * 1024;

bool tc_plan(int dtype, int ns, int nh, int64_t n_samples, TcDims* d);
size_t tc_workspace_bytes(const TcDims& d);
TcWork tc_layout(const TcDims& d, char* base);
// once per VMC step: BF16 tiles of T, T^T and Sigma^T
int tc_prepare_step(int dtype, const TcDims& d, int64_t n_samples, const uint32_t* bits, const void* tanh_theta,
                    const TcWork& w, cudaStream_t st);
// w_out = O v, partial[split] = O^H (wts (w - mean w) / Ns) with mean w = sum wts w / Ns (wts = 1 when
// w.wts is null), split over tc_matvec_nsplit(d) partial P-vectors; tanh_theta is T itself (float32 /
// complex64, Ns x nh), read by the fused kernel; cg_done (optional): a CG solve's converged flag, on
// which the kernels skip their work
int tc_matvec(int dtype, const TcDims& d, int64_t n_samples, const uint32_t* bits, const void* tanh_theta,
              const void* v, float2* w_out, void* partial, const TcWork& w, cudaStream_t st, bool build_vp = true,
              const double* cg_done = nullptr, BarCfg bc = BarCfg{0u, kGridBarLimit});
inline int tc_matvec_nsplit(const TcDims& d) { return d.sv ? d.sv_grid : d.nsplit; }
// w_out = O v only (builds the V' operand from v first)
int tc_ov(int dtype, const TcDims& d, int64_t n_samples, const uint32_t* bits, const void* tanh_theta, const void* v,
          float2* w_out, const TcWork& w, cudaStream_t st);
// partial[chunk] = O^H (wts (g - mean) * scale): gsum_n > 0 -> gsum_part holds gsum_n partial sums
// (mean = sum / Ns); gsum_n < 0 -> gsum_part[0] is the mean; gsum_part == nullptr -> no centring
int tc_ohu(int dtype, const TcDims& d, int64_t n_samples, const float2* g, const double2* gsum_part, int gsum_n,
           double scale, void* partial, const TcWork& w, cudaStream_t st);

// Writes the V' operand entries of one element of the direction vector (site i, hidden unit m;
// i == ns for the v_b part) straight into the chunked BF16 hi/lo tiles: used by the CG direction
// update so that no separate operand-building pass is needed.
#ifdef __CUDACC__
#include <cuda_bf16.h>
#include "umma.cuh"
__device__ __forceinline__ void tc_put_vp(const TcDims& d, uint16_t* vp, int n, int k, float x) {
  const uint16_t hi = __bfloat16_as_ushort(__float2bfloat16_rn(x));
  const uint16_t lo = __bfloat16_as_ushort(__float2bfloat16_rn(x - __bfloat162float(__ushort_as_bfloat16(hi))));
  const size_t term_bytes = (size_t)d.NB * d.KCH * 2;
  uint8_t* base = reinterpret_cast<uint8_t*>(vp) + (size_t)(k / d.KCH) * 2 * term_bytes;
  const uint32_t off = umma::kmajor_offset((uint32_t)n, (uint32_t)(k % d.KCH), (uint32_t)d.NB);
  *reinterpret_cast<uint16_t*>(base + off) = hi;
  *reinterpret_cast<uint16_t*>(base + term_bytes + off) = lo;
}
// Bz entry (row n, K index k): k-step k / 16 holds [hi tile | lo tile] of NZ rows x 16
__device__ __forceinline__ void tc_put_vz(const TcDims& d, uint16_t* vz, int n, int k, float x) {
  const uint16_t hi = __bfloat16_as_ushort(__float2bfloat16_rn(x));
  const uint16_t lo = __bfloat16_as_ushort(__float2bfloat16_rn(x - __bfloat162float(__ushort_as_bfloat16(hi))));
  const size_t tile_bytes = (size_t)d.NZ * 32;
  uint8_t* base = reinterpret_cast<uint8_t*>(vz) + (size_t)(k >> 4) * 2 * tile_bytes;
  const uint32_t off = umma::kmajor_offset((uint32_t)n, (uint32_t)(k & 15), (uint32_t)d.NZ);
  *reinterpret_cast<uint16_t*>(base + off) = hi;
  *reinterpret_cast<uint16_t*>(base + tile_bytes + off) = lo;
}
__device__ __forceinline__ void tc_put_vp_elem(const TcDims& d, uint16_t* vp, int i, int m, double vr) {
  if (d.ovz) {                                               // Bz: row m, K index i
    tc_put_vz(d, vp, m, i, (float)vr);
    return;
  }
  tc_put_vp(d, vp, i, m, (float)vr);                         // real RBM: row i, column m
}
__device__ __forceinline__ void tc_put_vp_elem(const TcDims& d, uint16_t* vp, int i, int m, double2 v) {
  const float vr = (float)v.x, vi = (float)v.y;
  if (d.ovz) {                                               // Bz: rows m (Re) and Mp + m (Im), K index i
    tc_put_vz(d, vp, m, i, vr);
    tc_put_vz(d, vp, d.Mp + m, i, vi);
    return;
  }
  if (d.splitc) {                                            // V'' rows: Re v, then Im v
    tc_put_vp(d, vp, i, m, vr);
    tc_put_vp(d, vp, d.Sp + i, m, vi);
    return;
  }
  tc_put_vp(d, vp, i, m, vr);                                // Re Y row: [Re v | -Im v]
  tc_put_vp(d, vp, i, d.Mp + m, -vi);
  tc_put_vp(d, vp, d.Sp + i, m, vi);                         // Im Y row: [Im v | Re v]
  tc_put_vp(d, vp, d.Sp + i, d.Mp + m, vr);
}
#endif
