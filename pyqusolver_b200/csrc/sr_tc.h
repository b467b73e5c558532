// Internal interface of the tensor-core SR matvec (sr_tc.cu) used by sr.cu.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

struct TcDims {
  int ns, nh;        // sites, hidden units
  int Kp;            // sites padded to 16 (K of the ov GEMM)
  int Mp;            // hidden units padded to 16 (N of one MMA)
  int Np;            // operand rows: 2*Mp (complex) or Mp (real)
  int KC;            // samples per ohu chunk (K of the ohu GEMM, multiple of 16)
  int im_off;        // TMEM column offset of the imaginary half
  int tmem_cols;     // TMEM columns allocated per CTA
  int n_tiles;       // ceil(Ns / 128)
  int n_chunks;      // ceil(Ns / KC)
  int ov_smem, ohu_smem;
};

struct TcWork {
  uint16_t* sig_rows;   // n_tiles x (128 x Kp) bf16, canonical K-major
  uint16_t* sig_cols;   // n_chunks x (128 x KC) bf16, canonical K-major
  uint16_t* bhi;        // Np x Kp bf16
  uint16_t* blo;
  double2* wsum;        // n_tiles partial sums of w = O v
  int* status;          // first error code of a bounded wait
};

constexpr size_t kTcSmemLimit = 220 * 1024;

bool tc_plan(int dtype, int ns, int nh, int64_t n_samples, TcDims* d);
size_t tc_workspace_bytes(const TcDims& d);
TcWork tc_layout(const TcDims& d, char* base);
int tc_prepare_step(const TcDims& d, int64_t n_samples, const uint32_t* bits, const TcWork& w, cudaStream_t st);
int tc_matvec(int dtype, const TcDims& d, int64_t n_samples, const uint32_t* bits, const void* tanh_theta,
              const void* v, float2* w_out, void* partial, const TcWork& w, cudaStream_t st);
// g centring: gsum_n > 0 -> gsum_part holds gsum_n partial sums (mean = sum / Ns);
// gsum_n < 0 -> gsum_part[0] is the mean; gsum_part == nullptr -> no centring
int tc_ohu(int dtype, const TcDims& d, int64_t n_samples, const uint32_t* bits, const void* tanh_theta,
           const float2* g, const double2* gsum_part, int gsum_n, double scale, void* partial, const TcWork& w,
           cudaStream_t st);
