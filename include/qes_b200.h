/*
 * qes_b200.h -- C ABI of the B200 RBM variational-Monte-Carlo library.
 *
 * One shared library (libqes_b200.so) exposes the hot path of QES's
 * neural-quantum-state VMC step for RBM ansaetze: Markov-chain sampling,
 * local energy, log-derivatives and the stochastic-reconfiguration solve.
 * Each entry point names the reference callable it replaces (file:line
 * within makskliczkowski/pyqusolver, Python/QES/...).
 *
 * Conventions
 *  - All array arguments are DEVICE pointers owned by the caller; the library
 *    never allocates.  Scratch space is passed in (size from *_workspace_bytes).
 *  - Every call is asynchronous on `stream` (a cudaStream_t, 0 = legacy default)
 *    and returns a status code; qes_last_error() gives the message.
 *  - dtype: QES_DTYPE_F32 (real RBM, float32) or QES_DTYPE_C64 (holomorphic
 *    complex RBM, complex64 interleaved re/im).
 *  - Spin configurations are bit-packed uint32 words, ceil(ns/32) per
 *    configuration: bit (i & 31) of word (i >> 5) is 1 for spin up
 *    (s = +0.5, sigma = +1).  Site order follows the lattice.
 *  - RBM: log psi(sigma) = sum_i a_i sigma_i + sum_m log cosh(theta_m),
 *    theta = W^T sigma + b, W row-major (ns x nh).  Flat parameter order is
 *    [a (ns), b (nh), W (ns*nh)].
 */
#ifndef QES_B200_H
#define QES_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define QES_OK 0
#define QES_ERR_ARG 1             /* bad shape / pointer / option              */
#define QES_ERR_CUDA 2            /* CUDA runtime error                        */
#define QES_ERR_WORKSPACE 3       /* workspace too small                       */
#define QES_ERR_NOT_CONVERGED 4   /* iterative solve hit maxiter               */
#define QES_ERR_TIMEOUT 5         /* a bounded device wait gave up             */
#define QES_ERR_SIZE 6            /* size beyond a compiled or static limit    */

#define QES_DTYPE_F32 0
#define QES_DTYPE_C64 1

#define QES_INIT_RND 0            /* independent random spins                  */
#define QES_INIT_RND_FIXED 1      /* fixed number of up spins, random order    */
#define QES_INIT_UP 2
#define QES_INIT_DOWN 3

#define QES_RULE_LOCAL 0          /* single spin flip                          */
#define QES_RULE_EXCHANGE 1       /* Sz-conserving neighbour exchange          */

#define QES_MOVE_FLIP1 0          /* flip site i                               */
#define QES_MOVE_PAIR_ANTI 1      /* flip i and j, active when sigma_i != sigma_j */
#define QES_MOVE_PAIR_PAR 2       /* flip i and j, active when sigma_i == sigma_j */

/* Last error message of the calling thread (static storage). */
const char* qes_last_error(void);
/* Library version: 100*major + minor. */
int qes_version(void);
/* Number of kernels this library launched in the process (reset != 0 zeroes
 * the counter after reading).  Host-side bookkeeping only. */
long long qes_launch_count(int reset);

/* ------------------------------------------------------------------------ */
/* Initial chain states.
 * Replaces QES/Solver/MonteCarlo/initialization/states.py:242-297
 * (_set_state_rand_fixed) and the RND initializer of the same file.
 * Philox stream: counter (chain, word|pos, 0, 1|2), key = seed.             */
int qes_init_chains(int kind, int n_up, uint64_t seed, int64_t chain_offset,
                    int n_chains, int ns, uint32_t* bits_out, void* stream);

/* ------------------------------------------------------------------------ */
/* Per-move ratio tables of the RBM (rebuilt after each parameter update).
 * For move k with sites (i, j) and kind:  D_k = W_i (FLIP1), W_i - W_j
 * (PAIR_ANTI), W_i + W_j (PAIR_PAR); Ct = cosh(2 D_km), St = sinh(2 D_km)
 * stored [m][k] (move_major = 0, local energy) or [k][m] (move_major = 1,
 * sampler); A[k] = a_i, a_i - a_j or a_i + a_j.
 * psi(s')/psi(s) = exp(-2 sigma_i A_k) prod_m (C_km - sigma_i tanh(theta_m) S_km).
 * Replaces the per-proposal ratio of net_rbm.log_psi_delta
 * (contract: Python/tests/nqs/test_rbm_fast_update.py:47-147).              */
int qes_rbm_move_tables(int dtype, int ns, int nh, const void* a, const void* W,
                        int n_moves, const int32_t* move_i, const int32_t* move_j,
                        const int32_t* move_kind, int move_major, void* Ct,
                        void* St, void* A, void* stream);

/* ------------------------------------------------------------------------ */
/* RBM forward on a batch of packed configurations: theta = W^T sigma + b,
 * tanh(theta) and log psi.  Any output pointer may be NULL.
 * Replaces the RBM apply (general_python net_rbm) as driven by
 * QES/Solver/MonteCarlo/vmc.py:1113-1164 (_batched_network_apply,
 * _init_logprobas_jax) and QES/NQS/nqs.py:1257-1280.                        */
int qes_rbm_forward(int dtype, int ns, int nh, int64_t n_samples,
                    const uint32_t* bits, const void* a, const void* b,
                    const void* W, void* theta_out, void* tanh_out,
                    void* logpsi_out, void* stream);

/* ------------------------------------------------------------------------ */
/* Metropolis sampler (persistent: one warp per chain).
 * Replaces VMCSampler._static_sample_jax / _run_mcmc_steps_jax
 * (QES/Solver/MonteCarlo/vmc.py:952-1103, 1186-1283) with the proposals of
 * QES/Solver/MonteCarlo/updates/spin_jax.py:51-158.
 * Schedule: therm_steps_total proposals, then num_samples records each
 * preceded by sweep_steps proposals.  Outputs are sample-major:
 * record r of chain c is row r*n_chains + c.                               */
typedef struct {
    int rule;                  /* QES_RULE_LOCAL / QES_RULE_EXCHANGE           */
    int ns, nh;
    int n_chains;
    int64_t chain_offset;      /* global id of chain 0 (Philox counter)        */
    int num_samples;
    int64_t therm_steps_total; /* proposals before the first record            */
    int sweep_steps;           /* proposals before each record                 */
    int recompute_every;       /* full theta recompute period (0 -> ns)        */
    float mu, beta;            /* acceptance: log u < min(beta*mu*Re dlogpsi, 0) */
    uint64_t seed;
    int deg;                   /* neighbour-table width (EXCHANGE)             */
} qes_sampler_config;

int qes_sampler_run(int dtype, const qes_sampler_config* cfg,
                    const void* a, const void* b, const void* W,
                    const void* flipCt, const void* flipSt,   /* tables of moves FLIP1 i=0..ns-1 */
                    const int32_t* nbr_table,                /* [ns*deg], -1 padded           */
                    const int32_t* nbr_pair,                 /* [ns*deg] pair index or -1     */
                    const int32_t* pair_i, const int32_t* pair_j, int n_pairs,
                    const void* pairCt, const void* pairSt,  /* PAIR_ANTI tables of the pairs */
                    uint32_t* chain_bits, uint64_t* chain_step,
                    int32_t* proposed, int32_t* accepted,
                    uint32_t* sample_bits, void* sample_logpsi, void* last_logpsi,
                    void* stream);

/* As qes_sampler_run with one beta per chain (chain_beta[n_chains], float32;
 * cfg->beta is ignored): the replica slots of parallel tempering.          */
int qes_sampler_run_betas(int dtype, const qes_sampler_config* cfg, const float* chain_beta,
                          const void* a, const void* b, const void* W,
                          const void* flipCt, const void* flipSt, const int32_t* nbr_table,
                          const int32_t* nbr_pair, const int32_t* pair_i, const int32_t* pair_j,
                          int n_pairs, const void* pairCt, const void* pairSt,
                          uint32_t* chain_bits, uint64_t* chain_step, int32_t* proposed,
                          int32_t* accepted, uint32_t* sample_bits, void* sample_logpsi,
                          void* last_logpsi, void* stream);

/* Programmatic dependent launch of the conjugate-gradient kernels (process-wide,
 * default on): each kernel of a CG iteration may start its prologue and the
 * prefetch of the per-step operands while its predecessor drains, and waits in
 * the kernel for the predecessor's results.  0 turns it off (plain stream
 * order); results are the same either way.                                  */
int qes_set_pdl(int on);

/* Device-driven CG loop (process-wide, default on): after the first chunk of
 * check_every iterations, the remaining full chunks run in one launch of a
 * CUDA graph whose conditional WHILE node repeats the chunk until the
 * converged flag is set (or the iteration limit), instead of one host
 * round trip per chunk.  Where the driver rejects such a graph the chunks
 * stay host-driven.  0 turns it off; results are the same either way.      */
int qes_set_cg_device_loop(int enable);

/* Which sampler kernel runs a chain set whose theta caches live in registers
 * (process-wide): 0 = the uncapped kernel (up to 128 registers, 16 chains per
 * SM); 1 = the kernel capped at 72 registers (28 chains per SM) when that
 * needs fewer waves of resident chains and spills no more (default);
 * 2 = the capped kernel always.  Samples are the same in every mode.        */
int qes_sampler_set_capped(int mode);
/* Hidden layers wider than one warp's register cache (nh > 512 real, > 256
 * complex), process-wide: 1 (default) runs each chain on a block of 2, 4 or
 * 8 warps, every thread holding 16 (real) / 8 (complex) units of the chain's
 * theta cache in registers, so a proposal's whole table row is fetched in
 * one round trip and the log-ratio is summed over the warps in order
 * (nh up to 4096 real / 2048 complex); 0 runs one warp per chain with the
 * cache in shared memory (nh up to 2048 real / 512 complex).  The two modes
 * draw the same random numbers and differ only in float32 summation order.
 * No counterpart in the reference (its sampler re-evaluates the network).  */
int qes_sampler_set_wide(int on);

/* The sampler's tanh of its acceptance cache applied elementwise (y = tanh x,
 * n elements of dtype): hardware exponential / sine / cosine / reciprocal
 * approximations, absolute error a few 1e-7 away from the poles of complex
 * tanh.  Exposed so that the error bound can be checked against float64.    */
int qes_sampler_tanh_cache(int dtype, int64_t n, const void* x, void* y, void* stream);

/* Parallel tempering (QES/Solver/MonteCarlo/vmc.py:1289-1507).  Chains are
 * n_replicas slots x n_chains (chain index r * n_chains + c); chain_beta holds
 * each chain's current beta.  qes_pt_swap exchanges beta labels between
 * adjacent slots (r, r+1), r of one parity per round (Philox counter
 * (round, 0, 0, 4) picks the parity; pair r of chain c draws counter
 * (c, round, r, 5)), accepting iff log u < min((b_r - b_r+1) mu
 * (Re lpsi_r+1 - Re lpsi_r), 0); swaps_accepted[r] (optional) counts swaps.
 * qes_pt_collect copies, per chain c, the slot whose beta equals
 * target_beta (|diff| < 1e-5, the first such slot) into row c of out_bits /
 * out_logpsi.                                                              */
int qes_pt_swap(int dtype, int n_replicas, int n_chains, const void* logpsi, float* chain_beta, float mu,
                uint64_t seed, int64_t round, int* swaps_accepted, void* stream);
int qes_pt_collect(int dtype, int n_replicas, int n_chains, int ns, const float* chain_beta,
                   float target_beta, const uint32_t* chain_bits, const void* logpsi,
                   uint32_t* out_bits, void* out_logpsi, void* stream);

/* ------------------------------------------------------------------------ */
/* Hamiltonian lowered to moves (off-diagonal) and diagonal terms.
 * Off-diagonal move k contributes  conj(c_k(s)) psi(s')/psi(s)  with
 * conj(c_k(s)) = (coef[4k] + i coef[4k+1]) + sigma_i (coef[4k+2] + i coef[4k+3]).
 * Diagonal: sum zf_h[t] sigma_{zf_site[t]} + sum zz_J[t] sigma_{zz_i[t]} sigma_{zz_j[t]}
 * (0.5 / 0.25 spin factors and QES signs already folded in).
 * Replaces QES/Algebra/Hamil/hamil_energy_jax.py:428-576 and the model
 * term builders (transverse_ising.py:192-300, xxz.py:278-433, j1j2.py:119-295). */
typedef struct {
    int n_moves;
    const int32_t* move_i;
    const int32_t* move_j;
    const int32_t* move_kind;
    const float* move_coef;    /* [4*n_moves] */
    int n_zfield;
    const int32_t* zf_site;
    const float* zf_h;
    int n_zz;
    const int32_t* zz_i;
    const int32_t* zz_j;
    const float* zz_J;
} qes_hamiltonian;

/* Local energy E_loc(s) = sum_k conj(c_k) psi(s'_k)/psi(s), complex64 out.
 * tanh_theta: [n_samples][nh] from qes_rbm_forward; Ct/St/A: move tables of
 * the same Hamiltonian moves.  Replaces net_utils_jax.apply_callable_batched_jax
 * (contract: Python/tests/nqs/test_nqs_generic_config_and_learning.py:282-371)
 * as called by QES/NQS/src/nqs_kernels.py:294-375.                          */
int qes_local_energy_workspace_bytes(int dtype, int ns, int nh, int64_t n_samples,
                                     int n_moves, size_t* bytes);
int qes_local_energy(int dtype, int ns, int nh, int64_t n_samples,
                     const uint32_t* bits, const void* tanh_theta,
                     const qes_hamiltonian* ham, const void* Ct, const void* St,
                     const void* A, void* workspace, size_t workspace_bytes,
                     void* eloc_out, void* stream);

/* Allocation-free variant of qes_local_energy -- no counterpart in the
 * reference.  For callers that cannot allocate device memory (a fixed device
 * budget handed over at start-up, loops that cannot afford cudaMalloc's
 * implicit synchronisation, foreign-language hosts without a device
 * allocator): the scratch lives in a static 8 MiB device array inside the
 * library, resident on every GPU that loads it until process exit.
 * Limit: ceil(n_moves/32) * n_samples * 8 bytes <= QES_NOALLOC_ELOC_SCRATCH_BYTES,
 * else QES_ERR_SIZE.  The first call on each device looks up the array's
 * device address (cudaGetSymbolAddress) and caches it; make that first call
 * before any stream capture.  Calls share the array: calls that overlap on
 * the GPU race on it.  Calls no cudaMalloc/cudaFree.                      */
#define QES_NOALLOC_ELOC_SCRATCH_BYTES (8u << 20)
int qes_local_energy_noalloc(int dtype, int ns, int nh, int64_t n_samples,
                             const uint32_t* bits, const void* tanh_theta,
                             const qes_hamiltonian* ham, const void* Ct,
                             const void* St, const void* A, void* eloc_out,
                             void* stream);

/* ------------------------------------------------------------------------ */
/* Energy statistics in float64 (compensated): out = [mean_re, mean_im, var, std]
 * with weights probs (NULL = uniform).  Replaces the mean/std of
 * QES/NQS/src/tdvp.py:1075-1076 and the estimator statistics.              */
int qes_loss_stats_workspace_bytes(int64_t n_samples, size_t* bytes);
int qes_loss_stats(int64_t n_samples, const void* eloc, const float* probs,
                   double* out, void* workspace, size_t workspace_bytes, void* stream);

/* Step diagnostics in float64: out = [r_hat, sigma2].  r_hat is the
 * Gelman-Rubin statistic of Re E_loc split into n_chains contiguous blocks
 * (NaN when n_chains <= 1, n_samples <= n_chains, n_samples % n_chains != 0
 * or a block has one sample); sigma2 = var(Re E_loc), uniform weights,
 * ddof 0.  Replaces TDVP._compute_step_rhat and the sigma2 of
 * QES/NQS/src/tdvp.py:1487-1518, 1642-1643.                                */
int qes_loss_rhat_workspace_bytes(int64_t n_samples, int n_chains, size_t* bytes);
int qes_loss_rhat(int64_t n_samples, int n_chains, const void* eloc, double* out,
                  void* workspace, size_t workspace_bytes, void* stream);

/* ------------------------------------------------------------------------ */
/* Per-sample log-derivatives O (rows of P = ns + nh + ns*nh, leading dim ldo):
 * O_a = sigma_i, O_b = tanh theta_m, O_W = sigma_i tanh theta_m.
 * Replaces compute_gradients_batched / log_derivative_jax
 * (QES/NQS/src/nqs_kernels.py:212-259, QES/NQS/nqs.py:2134-2188).          */
int qes_rbm_log_derivatives(int dtype, int ns, int nh, int64_t n_samples,
                            const uint32_t* bits, const void* tanh_theta,
                            void* O_out, int64_t ldo, void* stream);

/* ------------------------------------------------------------------------ */
/* Stochastic reconfiguration with the RBM's structured O (never materialised):
 *   (O_c^H O_c / Ns + shift) x = F,  F = O_c^H E_c / Ns,  x <- rhs_prefactor x.
 * Vectors are float64 (real RBM) or complex128 (complex RBM), length P.
 * Replaces TDVP.get_tdvp_standard / _solve_prepare_matvec / solve
 * (QES/NQS/src/tdvp.py:1056-1197,1524-1609) with SciPy-style CG
 * (||r|| <= max(rtol ||b||, atol); nqs.py:3014 default 'scipy_cg').        */
typedef struct {
    double shift;
    double rtol;
    double atol;
    int maxiter;
    int check_every;           /* host convergence check period (iterations) */
    double rhs_prefactor;
    int precond;               /* QES_PRECOND_NONE, or QES_PRECOND_JACOBI: CG with
                                  M = 1 / diag(S + shift), diag(S)_k = mean|O_k|^2 -
                                  |mean O_k|^2 (weighted), SciPy's cg(M=...) semantics
                                  (the stopping rule stays on ||r||).  The CG solve only;
                                  MinSR and the batched CG take QES_PRECOND_NONE.
                                  Replaces the 'jacobi' pre_solver / sr_precond of
                                  QES/NQS/src/tdvp.py:332,686-710.                    */
    int skip_true_residual;    /* nonzero: the CG / MINRES solve does not recompute
                                  ||F - (S + shift) x|| / ||F|| after it ends (one
                                  matvec and a host read fewer; result->true_residual
                                  = -1).  0 (a zero-initialised struct): computed.   */
} qes_sr_options;

#define QES_PRECOND_NONE 0
#define QES_PRECOND_JACOBI 1

typedef struct {
    int iterations;
    int converged;             /* SciPy's rule met by CG's recursive residual */
    double residual;           /* recursive residual norm at exit */
    double rhs_norm;
    double e_mean_re, e_mean_im;
    double true_residual;      /* ||F - (S + shift) x|| / ||F|| recomputed with one more
                                  matvec after the solve (-1: not computed).  With float32
                                  or BF16-split contractions it levels off near their
                                  rounding (~1e-6-1e-5) while the recursive residual keeps
                                  falling; no counterpart in the reference (float64 SR). */
    double acond;              /* MINRES: max / min of the rotated diagonal (gamma_k), the
                                  estimate of cond(S + shift) that MINRES-QLP compares
                                  with its switch threshold; -1 for the other solvers.   */
} qes_sr_result;

int qes_sr_workspace_bytes(int dtype, int ns, int nh, int64_t n_samples, size_t* bytes);

/* Matvec implementation of the SR calls in this process: 0 = 5th-generation
 * tensor cores (tcgen05, BF16 hi/lo split, FP32 accumulate) when the tiling
 * fits (ns <= 511, V' <= 512 rows, shared memory), CUDA cores otherwise
 * (default); 1 = CUDA cores only (float32); 2 = tensor cores required
 * (QES_ERR_SIZE when the shapes do not allow them); 3 = CUDA cores with
 * float64 contractions of the same float32 T (the reference's SR precision:
 * it promotes O to float64, tdvp.py:827-858), a slow reference form for
 * accuracy checks (not MinSR).  No counterpart in the reference
 * (its SR runs on XLA).  qes_sr_force / qes_sr_matvec synchronise the stream
 * when the tensor-core path ran, to report bounded-wait time-outs.          */
int qes_set_sr_impl(int impl);
/* *uses = 1 when the SR calls for these shapes run on the tensor cores under
 * the current qes_set_sr_impl setting, else 0.                             */
int qes_sr_uses_tensor_cores(int dtype, int ns, int nh, int64_t n_samples, int* uses);
/* Tiling of the tensor-core path for these shapes (for roofline accounting):
 * out = [uses, big, KC, n_chunks, nsplit, n_tiles, Kd, NB, Np, MT, NC, NR,
 * nnc, SPC, ov_stages, cl, sv, sv_grid, ovz] (first n_out entries); cl = 2
 * when the O^H u CTAs run as pairs that add their partials on chip; sv = 1
 * when the matvec runs as the fused S v kernel of sv_grid CTAs (one partial
 * each); ovz = 1 when O v runs through z = Sigma V (qes_sr_set_ovz).       */
int qes_sr_tc_plan(int dtype, int ns, int nh, int64_t n_samples, int32_t* out, int n_out);
/* Tiling of the tensor-core O^H u in this process: mode 0 = automatic (the
 * single-M-tile kernel when the shapes allow it), 1 = single-M-tile kernel
 * only, 2 = M/N-tiled kernel; nc = hidden units per N chunk (multiple of 16,
 * 0 = largest that fits TMEM); ctas = target CTA count (0 = 296).          */
int qes_sr_set_tiling(int mode, int nc, int ctas);
/* O^H u of the single-M-tile kernel as thread-block clusters of two CTAs that
 * add their split-K partials through distributed shared memory before writing
 * one per pair (1, where the W block fits the staging buffers) or one partial
 * per CTA (0, the default: the pairs measured slower on B200).  Same sums in a
 * fixed order either way.                                                  */
int qes_sr_set_ohu_pairs(int on);
/* The tensor-core S v of single-M-tile problems as one cooperative launch
 * (1): each CTA computes O v for its 128-sample tiles, a grid barrier gives
 * every CTA the weighted mean of O v, and the same CTA then accumulates
 * O^H u of its tiles in TMEM (Q = conj(t) u built from the float32 T) and
 * writes one partial P-vector; or as the two kernels O v and O^H u (0, the
 * default: measured faster on B200).  Same operator, different float32
 * summation order.                                                        */
int qes_sr_set_fused_sv(int on);
/* Complex O v on the tensor cores when 2 (sites + 1) <= 256 (1):
 * two products T_re V''^T and T_im V''^T into two TMEM accumulators, V'' =
 * [Re v ; Im v] over the hidden units, combined in the epilogue (Re Y =
 * D1_re - D2_im, Im Y = D1_im + D2_re); every O v CTA then reads half the
 * direction-operand bytes of the single product over K = [Re t | Im t]
 * against [Re v | -Im v ; Im v | Re v] (0, the default: measured as fast,
 * O v is bound by its MMAs).  Same products, different
 * float32 summation order.  Takes the fused S v kernel out of the plan
 * (it reads the single-product operand).                                  */
int qes_sr_set_ov_split(int on);
/* O v through z = Sigma V (1, the default where the operands fit: NZ = 2 Mp
 * (complex) or Mp (real) hidden-unit rows <= 512 and 128 x Kz spins plus the
 * whole NZ x Kz direction operand within shared memory, Kz = sites + 1 padded
 * to 16): A = the +-1 spins and a ones column (exact in BF16), B = the
 * direction's W block and v_b (BF16 hi + lo), so the MMAs yield
 * z_s = sigma_s^T V + v_b for every hidden unit; the epilogue forms
 * (O v)_s = sum_m t_sm z_sm + sigma_s . v_a with t in float32 read from
 * tanh_theta itself.  0: the product over the hidden axis (T as A in hi/lo
 * against V').  Same operator; the hi/lo split touches v only.  Takes the
 * fused S v kernel and the split-complex product out of the plan.          */
int qes_sr_set_ovz(int on);
/* tc_ovz_kernel's CTAs pull their 128-sample tile of the transposed T into
 * L2 (cp.async.bulk.prefetch.L2) before they wait on the previous kernel
 * of the CG chain (1), or not (0, the default: measured the same, 42.1 vs
 * 42.3 us per 10x10 CG iteration, T already stays in L2).  A hint: results
 * are the same either way.                                                 */
int qes_sr_set_prefetch(int on);
/* CG iteration chunks replayed as CUDA graphs on a private stream (1, the
 * default) or launched one by one on the caller's stream (0).              */
int qes_set_cg_graphs(int enable);
/* The vector part of each CG iteration (split-partial reduction, x/r and
 * direction updates) as one cooperative kernel with two bounded grid
 * barriers: 2 = always, 1 = when its grid is at most 160 CTAs (the default:
 * parameter vectors up to a few thousand entries, where launch latency
 * dominates), 3 = always with one CTA per SM (fewer grid-barrier arrivals),
 * 0 = never (three kernels).                                               */
int qes_set_cg_fused(int mode);
/* CG steps in the Chronopoulos-Gear form on the kernel-chain path (1; for
 * the unpreconditioned CG): the matvec is applied to r_k, its
 * split reduction also sums |r_k|^2 with r_k^H A r_k, and its last block
 * forms beta_k = |r_k|^2 / |r_{k-1}|^2, alpha_k = |r_k|^2 / (r_k^H A r_k -
 * beta_k |r_k|^2 / alpha_{k-1}) and the convergence test on |r_k|^2; one
 * kernel then updates p, s = A p (by recurrence), x and r: one grid-wide
 * reduction and one kernel per step fewer than the standard form (0, the
 * default: the matvec of p, then the x/r update with its |r|^2 reduction,
 * then the p update).  The same Krylov iterates in exact arithmetic and the
 * same stopping rule on the residual vector's norm (Chronopoulos and Gear,
 * J. Comput. Appl. Math. 25 (1989)); p^H A p is formed from the vectors
 * (bilinear in the recurrences), not from orthogonality.  Measured on B200:
 * 10x10 Heisenberg CG iteration 43.3 -> 40.3 us at the same iteration count,
 * but the recurrence of s carries the float32 / BF16-split operator's
 * rounding forward, and a strongly rank-deficient system (20x20 TFIM, 256
 * samples, 642,000 parameters) did not converge where the standard form
 * does, so it is off by default.  With the Jacobi preconditioner and in the
 * fused cooperative vector kernel (qes_set_cg_fused) the standard form
 * runs.                                                                    */
int qes_set_cg_single_reduction(int on);
/* The split reduction of the SR matvec (the sum of the split-K partial
 * P-vectors that the O^H u kernels write, + shift p and the CG dot products)
 * with each block's column slices of every partial moved into shared memory
 * by bulk copies under one mbarrier (1, where the slices fit 88 KB: two
 * blocks per SM), or loaded by the threads in batches of 16-byte loads (0,
 * the default: measured faster on B200, 12.8 against 16.8 us per launch on
 * the 10x10 workload, where the bulk form issues 147 small copies per
 * block).  Same sums in the same order: bit-identical results.            */
int qes_set_reduce_bulk(int on);
/* The x/r update and the direction update of a standard CG step in one
 * launch (1, the default on the kernel-chain path): phase 1 updates x and r
 * and sums |r|^2 per block, a bounded grid barrier, then every CTA sums the
 * partials in the same order as the two-kernel form and updates its slice
 * of p and the tensor-core operand tiles (0: cg_xr then cg_p).  Bit-
 * identical results; one launch boundary and one last-block step fewer.
 * The fused cooperative vector kernel (qes_set_cg_fused) and the
 * Chronopoulos-Gear steps take precedence where they are selected.         */
int qes_set_cg_xrp(int on);
/* The fused cooperative vector kernel (qes_set_cg_fused) launched by
 * programmatic dependent launch (1, the default) instead of as a cooperative
 * launch (0): its grid, sized within residency, is co-resident once every
 * CTA has run the trigger at its entry, and its prologue overlaps the O^H u
 * kernel's tail (TFIM-16 CG iteration 18.8 -> 18.3 us).  Same kernel, same
 * sums: bit-identical results.                                            */
int qes_set_cg_fused_pdl(int on);
/* Test hook of the fused CG kernel's grid barriers (no reference
 * counterpart): (1, polls) makes every barrier wait for one arrival that
 * never comes and give up after `polls` polls, so a solve returns
 * QES_ERR_TIMEOUT at its next status check; (0, 0) restores the normal
 * barriers.  Process-wide; meant for tests of the time-out path only.      */
int qes_sr_set_barrier_test(unsigned int extra_arrivals, unsigned int poll_limit);

/* RBM forward on the tensor cores: theta = Sigma W + b with W split into
 * three BF16 terms (exact for float32 W) and float32 accumulation; outputs
 * as qes_rbm_forward.  Workspace from qes_rbm_forward_tc_workspace_bytes
 * (QES_ERR_SIZE when the shapes are outside its limits).  Replaces the
 * network apply of QES/Solver/MonteCarlo/vmc.py:1113-1147 for a batch.      */
int qes_rbm_forward_tc_workspace_bytes(int dtype, int ns, int nh, int64_t n_samples, size_t* bytes);
int qes_rbm_forward_tc(int dtype, int ns, int nh, int64_t n_samples, const uint32_t* bits,
                       const void* a, const void* b, const void* W, void* theta_out,
                       void* tanh_out, void* logpsi_out, void* workspace, size_t workspace_bytes,
                       void* stream);
/* Keep the tensor-core operand tiles resident in L2 across CG iterations
 * through a persisting access-policy window on the solve's streams (1; the
 * window and the persisting lines are released after each solve) or not (0,
 * the default: the tiles already stay in L2 between the iterations of the
 * bench workloads).  Numerical results do not depend on it.               */
int qes_set_l2_persist(int enable);

/* Per-kernel CUDA-event timing of the SR matvec halves, for measurement:
 * while enabled, every launch of class k (0: O v, 1: O^H u, 2: split
 * reduction, 3: dense Gram, 4: dense Cholesky, the whole factorisation,
 * 5: the fused S v kernel)
 * is bracketed by two events on its launch stream and CG graphs
 * are bypassed.  qes_profile_read synchronises the device and returns the
 * accumulated milliseconds and launch counts (reset != 0 zeroes them).
 * No counterpart in the reference (it has no per-kernel timing).          */
int qes_profile_enable(int enable);
int qes_profile_read(int reset, double* total_ms, long long* counts, int n);

/* F = O_c^H E_c / Ns (force) and the matvec y = (O_c^H O_c / Ns + shift) v. */
int qes_sr_force(int dtype, int ns, int nh, int64_t n_samples,
                 const uint32_t* bits, const void* tanh_theta, const void* eloc,
                 void* force_out, void* workspace, size_t workspace_bytes, void* stream);
int qes_sr_matvec(int dtype, int ns, int nh, int64_t n_samples,
                  const uint32_t* bits, const void* tanh_theta, double shift,
                  const void* v, void* y_out, void* workspace,
                  size_t workspace_bytes, void* stream);
int qes_sr_solve_cg(int dtype, int ns, int nh, int64_t n_samples,
                    const uint32_t* bits, const void* tanh_theta, const void* eloc,
                    const qes_sr_options* opt, void* x_out, qes_sr_result* result,
                    void* workspace, size_t workspace_bytes, void* stream);
/* The same three with per-sample weights `probs` (float32, normalised to sum
 * Ns, as VMCSampler returns them when 1/logprob_fact != mu beta;
 * QES/Solver/MonteCarlo/vmc.py:1173-1184): means are weighted,
 * <X> = sum_s p_s X_s / Ns, and every sample sum carries p_s:
 *   F = O^H (p (E - <E>)) / Ns,  S v = O^H (p (O v - <O v>)) / Ns,
 * which is O_c^H diag(p) O_c / Ns with O_c centred by the weighted mean.
 * The weighting of the SR sums is this library's reading of the reference
 * (its SR module is not in the snapshot; its sampler produces the weights
 * and its estimator takes them).  probs = NULL is the unweighted call.      */
int qes_sr_force_weighted(int dtype, int ns, int nh, int64_t n_samples, const uint32_t* bits,
                          const void* tanh_theta, const void* eloc, const float* probs,
                          void* force_out, void* workspace, size_t workspace_bytes, void* stream);
int qes_sr_matvec_weighted(int dtype, int ns, int nh, int64_t n_samples, const uint32_t* bits,
                           const void* tanh_theta, const float* probs, double shift, const void* v,
                           void* y_out, void* workspace, size_t workspace_bytes, void* stream);
int qes_sr_solve_cg_weighted(int dtype, int ns, int nh, int64_t n_samples, const uint32_t* bits,
                             const void* tanh_theta, const void* eloc, const float* probs,
                             const qes_sr_options* opt, const void* x0, void* x_out,
                             qes_sr_result* result, void* workspace, size_t workspace_bytes,
                             void* stream);
/* The same system solved by MINRES (Paige-Saunders recurrences as in SciPy's
 * minres, no preconditioner): same force, matvec, workspace, x0 and
 * rhs_prefactor handling as the CG; it stops when the recurrence's residual
 * norm phibar <= max(rtol ||F||, atol) (the CG's rule) and reports the
 * condition estimate in result->acond.  Replaces the 'minres' / 'minres_qlp'
 * lin_solver of QES/NQS/__init__.py:406 and tdvp.py:322-350 (MINRES-QLP
 * follows MINRES until the condition estimate passes its switch threshold,
 * ~1e7 in the published algorithm; the caller can compare result->acond). */
int qes_sr_solve_minres_weighted(int dtype, int ns, int nh, int64_t n_samples, const uint32_t* bits,
                                 const void* tanh_theta, const void* eloc, const float* probs,
                                 const qes_sr_options* opt, const void* x0, void* x_out,
                                 qes_sr_result* result, void* workspace, size_t workspace_bytes,
                                 void* stream);
/* As qes_sr_solve_cg with an initial guess x0 (device, P float64 / complex128)
 * of the unscaled system (S + shift) x = F, i.e. a previous x_out divided by
 * rhs_prefactor; r0 = F - (S + shift) x0 costs one extra matvec and the stop
 * rule stays ||r|| <= max(rtol ||F||, atol).  x0 = NULL starts from zero.
 * Replaces the initial-guess handling of TDVP.solve (sr_lin_x0 and
 * use_old_result, QES/NQS/src/tdvp.py:1346-1380).                          */
int qes_sr_solve_cg_x0(int dtype, int ns, int nh, int64_t n_samples,
                       const uint32_t* bits, const void* tanh_theta, const void* eloc,
                       const qes_sr_options* opt, const void* x0, void* x_out,
                       qes_sr_result* result, void* workspace, size_t workspace_bytes,
                       void* stream);

/* Formed SR matrix (TDVP sr_form_matrix=True; QES/NQS/src/tdvp.py:340,455
 * and the covariance of get_tdvp_standard :1113-1117) and its direct solve.
 * S = O_c^H diag(p) O_c / Ns (p = probs normalised to sum Ns, NULL =
 * uniform; O_c centred by the weighted mean) is formed on the tensor cores:
 * the centred O as BF16 hi/lo tiles, hi*hi + hi*lo + lo*hi tcgen05 MMAs with
 * FP32 accumulation in TMEM over the samples, combined into float64.
 * qes_sr_gram writes S (P x P row-major, full Hermitian, float64 /
 * complex128) to s_out.  qes_sr_solve_dense factorises S + shift = L L^H in
 * float64 (blocked Cholesky) and solves for x = rhs_prefactor (S + shift)^-1 F;
 * result: iterations 0, converged 0 and QES_ERR_NOT_CONVERGED when S + shift
 * is not positive definite in float64, true_residual = ||F - (S + shift) x||
 * / ||F|| with the formed S.  Memory grows as P^2: QES_ERR_SIZE when the
 * workspace would exceed 100 GB (use the matrix-free qes_sr_solve_cg).
 * Workspace from qes_sr_dense_workspace_bytes (gram_only != 0: the smaller
 * workspace of qes_sr_gram).                                               */
int qes_sr_dense_workspace_bytes(int dtype, int ns, int nh, int64_t n_samples, int gram_only, size_t* bytes);
int qes_sr_gram(int dtype, int ns, int nh, int64_t n_samples, const uint32_t* bits,
                const void* tanh_theta, const float* probs, void* s_out, void* workspace,
                size_t workspace_bytes, void* stream);
int qes_sr_solve_dense(int dtype, int ns, int nh, int64_t n_samples, const uint32_t* bits,
                       const void* tanh_theta, const void* eloc, const float* probs,
                       const qes_sr_options* opt, void* x_out, qes_sr_result* result,
                       void* workspace, size_t workspace_bytes, void* stream);

/* Vector-Jacobian product of log psi for the hand-written backward:
 * grad = O^H g  (g: complex64 per sample; real part used for a real RBM),
 * float64/complex128 out, length P.  Replaces jax.vjp of the RBM apply
 * behind compute_gradients_batched (QES/NQS/src/nqs_kernels.py:212-259).
 * Workspace: qes_sr_workspace_bytes.                                        */
int qes_rbm_logpsi_vjp(int dtype, int ns, int nh, int64_t n_samples,
                       const uint32_t* bits, const void* tanh_theta, const void* g,
                       void* grad_out, void* workspace, size_t workspace_bytes,
                       void* stream);

/* Euler / SGD update in float64: master += lr * x; params = (float) master.
 * Replaces NQSTrainer._apply_parameter_update (QES/NQS/src/nqs_train.py:1235-1262). */
int qes_param_update(int dtype, int64_t n_params, double lr, const void* x,
                     void* master, void* params, void* stream);

/* MinSR (QES/NQS/src/tdvp.py:1199-1226, 1393-1408): solve
 * (O_c O_c^H / Ns + shift) y = E_c / Ns by CG in sample space (float64,
 * SciPy's stopping rule on that system) and return x = rhs_prefactor O_c^H y
 * (length P).  Matrix-free: each iteration applies O_c^H then O_c with the
 * kernels of qes_sr_matvec (tensor cores under qes_set_sr_impl as there).
 * Workspace from qes_sr_minsr_workspace_bytes.                             */
int qes_sr_minsr_workspace_bytes(int dtype, int ns, int nh, int64_t n_samples, size_t* bytes);
int qes_sr_solve_minsr(int dtype, int ns, int nh, int64_t n_samples, const uint32_t* bits,
                       const void* tanh_theta, const void* eloc, const qes_sr_options* opt,
                       void* x_out, qes_sr_result* result, void* workspace, size_t workspace_bytes,
                       void* stream);

/* Replica swap of the sites in mask_words (packed like a configuration) between
 * two sample batches: out_a = (a outside A, b inside A), out_b the opposite.
 * The Renyi-2 swap estimator of QES/NQS/src/nqs_entropy.py:311-460.        */
int qes_swap_region(int64_t n_samples, int ns, const uint32_t* mask_words, const uint32_t* bits_a,
                    const uint32_t* bits_b, uint32_t* out_a, uint32_t* out_b, void* stream);

/* ------------------------------------------------------------------------ */
/* Exact ground energy (the ED reference of the energy-error metric): Lanczos
 * over the full 2^ns S^z product basis (ns <= 32; basis bit i = site i,
 * 1 = up) with the Hamiltonian applied matrix-free from `ham` (the same
 * lowered terms the local energy reads; real matrix elements only).
 * y = H x for qes_ed_matvec.  Lanczos stops when the lowest Ritz value
 * changes by <= tol * max(1, |E|) between iterations (QES_ERR_NOT_CONVERGED
 * after max_iter).  Replaces model.diagonalize(method='lanczos')
 * (QES/Algebra/hamil.py:1809; its solver lives in the absent eigen module). */
int qes_ed_workspace_bytes(int ns, size_t* bytes);
int qes_ed_matvec(int ns, const qes_hamiltonian* ham, const double* x, double* y, void* stream);
int qes_ed_lanczos(int ns, const qes_hamiltonian* ham, int max_iter, double tol, uint64_t seed,
                   double* e0_out, int* iterations_out, void* workspace, size_t workspace_bytes,
                   void* stream);
/* Lanczos in one S^z sector (n_up up spins) of an S^z-conserving Hamiltonian (anti-parallel pair
 * moves only), optionally restricted further to one spin-flip parity (+1 / -1; needs ns = 2 n_up
 * and no z field): the basis is indexed by the colex rank of the bit-packed state (the lower
 * ns - 1 sites with parity, a state and its flip sharing one basis vector), so no index table is
 * stored and the vectors hold C(ns, n_up) (or C(ns - 1, n_up)) float64 entries.  ns <= 62,
 * n_up <= 32.  Workspace from qes_ed_sector_workspace_bytes; qes_ed_sector_dim gives the
 * dimension.  Replaces model.diagonalize(method='lanczos') on a symmetry sector
 * (QES/Algebra/hamil.py:1809+, QES/Algebra/Hamil/hamil_diag_engine.py:176-305).              */
int qes_ed_sector_dim(int ns, int n_up, int parity, uint64_t* dim);
int qes_ed_sector_workspace_bytes(int ns, int n_up, int parity, size_t* bytes);
int qes_ed_lanczos_sector(int ns, int n_up, int parity, const qes_hamiltonian* ham, int max_iter,
                          double tol, uint64_t seed, double* e0_out, int* iterations_out,
                          void* workspace, size_t workspace_bytes, void* stream);
/* Lanczos in a momentum sector of a translation-invariant S^z-conserving Hamiltonian on an
 * lx x ly periodic lattice (site x + lx*y; a chain is ly = 1, lx*ly <= 62): the states with n_up
 * up spins reduced by the lx*ly translations and, with parity = +1 / -1 (ns = 2 n_up, no z field),
 * the spin flip; momentum 0 (kx/ky = 0) or pi (= 1, even side) per axis, the real characters of
 * QES/Algebra/Symmetries/translation.py:470-519 (sector index 0 or L/2).  Basis: the orbit
 * minima, listed on the device by two enumeration passes over the C(ns, n_up) (C(ns - 1, n_up)
 * with the flip; at most 2^37) colex ranks.  Call qes_ed_symm_dim (workspace from
 * qes_ed_symm_workspace_bytes with dim = 0) for the dimension, then qes_ed_symm_workspace_bytes
 * with it (≈ 32 (dim + 1) + C/8 bytes for C ranks) for qes_ed_lanczos_symm.  The Hamiltonian is
 * checked on the host: anti-parallel pair moves with real coefficients, bonds and fields that map
 * onto themselves under T(1, 0) and T(0, 1) (else QES_ERR_ARG).  dim_out (optional) receives
 * the sector dimension.  Replaces model.diagonalize(method='lanczos') in a symmetry sector of a
 * HilbertSpace with translation and parity symmetries (QES/Algebra/hamil.py:1809+,
 * QES/Algebra/Symmetries/momentum_sectors.py).                                               */
int qes_ed_symm_workspace_bytes(int lx, int ly, int n_up, int parity, int kx, int ky, uint64_t dim,
                                size_t* bytes);
int qes_ed_symm_dim(int lx, int ly, int n_up, int parity, int kx, int ky, uint64_t* dim,
                    void* workspace, size_t workspace_bytes, void* stream);
int qes_ed_lanczos_symm(int lx, int ly, int n_up, int parity, int kx, int ky, const qes_hamiltonian* ham,
                        int max_iter, double tol, uint64_t seed, double* e0_out, int* iterations_out,
                        uint64_t* dim_out, void* workspace, size_t workspace_bytes, void* stream);

/* ------------------------------------------------------------------------ */
/* Batched independent problems.  Many (RBM, Hamiltonian, chain set) triples
 * of uneven size advance together: every phase of the VMC step is one
 * launch over all problems.  The reference runs one NQS per problem
 * (QES/NQS/nqs.py:241); these calls replace a Python loop over such objects.
 *
 * `inst` is a DEVICE array of n_inst descriptors.  Buffers are the
 * concatenation of the per-problem buffers; each offset below is in elements
 * (words for bit buffers) of the buffer it names.  Work lists are DEVICE
 * arrays of int32 quadruples built by the host from the descriptors (the
 * Python host orders them by decreasing cost); their meaning is given per
 * call.  Problem b's sampler is bit-identical to qes_sampler_run with
 * seed = inst[b].seed and chain_offset = 0.                                 */
typedef struct {
    int32_t ns, nh;                 /* sites, hidden units                          */
    int32_t n_moves, n_zz, n_zfield;/* lowered Hamiltonian sizes                    */
    int32_t n_chains, num_samples;  /* chains; recorded samples per chain per call  */
    int32_t sweep_steps;            /* proposals between recorded samples           */
    int64_t therm_steps_total;      /* proposals before the first record            */
    uint64_t seed;                  /* Philox key of this problem                   */
    int64_t param_off;              /* [a, b, W] in params and in every P-vector    */
    int64_t chain_off;              /* chain_step / proposed / accepted / last_logpsi */
    int64_t chain_word_off;         /* chain_bits                                   */
    int64_t sample_off;             /* sample rows: logpsi, eloc (rows = n_chains*num_samples, sample-major) */
    int64_t sample_word_off;        /* sample_bits                                  */
    int64_t tanh_off;               /* tanh(theta) rows x nh                        */
    int64_t flip_off;               /* single-flip tables, ns x nh (sampler)        */
    int64_t move_table_off;         /* local-energy tables, nh x n_moves            */
    int64_t move_off, zz_off, zf_off; /* move / zz / z-field arrays and move A values */
    int64_t eloc_part_off;          /* local-energy partials, ceil(n_moves/32) x rows */
    int64_t sr_part_off;            /* SR split partials, ceil(rows/256) x P        */
} qes_batch_instance;

/* ns x nh single-flip tables (mode 0, items (b, first element / 256, 0, 0),
 * tables at flip_off, move-major) or the nh x n_moves local-energy tables
 * (mode 1, tables at move_table_off, m-major, A at move_off) of every
 * problem.  Same values as qes_rbm_move_tables.                            */
int qes_batch_move_tables(int dtype, int n_inst, const qes_batch_instance* inst, int mode, int n_items,
                          const int32_t* items, const void* params, const int32_t* move_i,
                          const int32_t* move_j, const int32_t* move_kind, void* Ct, void* St, void* A,
                          void* stream);
/* Single-flip Metropolis sampling of every problem's chains in one
 * persistent launch: n_blocks blocks of warps_per_block warps take chains
 * (items (b, chain, 0, 0)) from a device queue; counter = 4 bytes of device
 * scratch; max_nh = largest nh (sizes the register-resident theta cache).
 * therm_steps_total is honoured when thermalize != 0.                      */
int qes_batch_sampler_run(int dtype, int n_inst, const qes_batch_instance* inst, int max_nh,
                          int n_items, const int32_t* items, int warps_per_block, int n_blocks, int thermalize,
                          float mu, float beta, int recompute_every, const void* params,
                          const void* flipCt, const void* flipSt, uint32_t* chain_bits,
                          uint64_t* chain_step, int32_t* proposed, int32_t* accepted,
                          uint32_t* sample_bits, void* sample_logpsi, void* last_logpsi,
                          unsigned int* counter, void* stream);
/* tanh(theta) (at tanh_off) and log psi (at sample_off, may be NULL) of the
 * recorded samples; items (b, sample block of 16, 0, 0).                   */
int qes_batch_rbm_forward(int dtype, int n_inst, const qes_batch_instance* inst, int n_items,
                          const int32_t* items, const void* params, const uint32_t* sample_bits,
                          void* tanh_out, void* logpsi_out, void* stream);
/* E_loc of every sample; move items (b, move block of 32, sample block of
 * 32, 0), reduce items (b, sample block of 256, 0, 0); partial = scratch of
 * sum_b ceil(n_moves/32) * rows complex64.                                 */
int qes_batch_local_energy(int dtype, int n_inst, const qes_batch_instance* inst, int n_move_items,
                           const int32_t* move_items, int n_red_items, const int32_t* red_items,
                           const uint32_t* sample_bits, const void* tanh_theta, const int32_t* move_i,
                           const int32_t* move_j, const int32_t* move_kind, const float* move_coef,
                           const void* Ct, const void* St, const void* A, const int32_t* zf_site,
                           const float* zf_h, const int32_t* zz_i, const int32_t* zz_j, const float* zz_J,
                           void* partial, void* eloc_out, void* stream);
/* out[b] = [mean_re, mean_im, var, std] of problem b's E_loc in float64.   */
int qes_batch_loss_stats(int n_inst, const qes_batch_instance* inst, const void* eloc, double* out,
                         void* stream);
/* Per-problem SR solve (S_b + shift) x_b = F_b by CG, all problems in
 * lockstep launches, each frozen at its own convergence; x at param_off
 * (float64 / complex128), scaled by rhs_prefactor.  ov items (b, first
 * row, rows <= 64, 0); ohu items (b, split of 256 samples, 0, 0).  Each
 * problem needs ns * nh <= 16384 (real) / 8192 (complex) and nh <= 512
 * (QES_ERR_SIZE otherwise): the batch is meant for many small problems.  sr_part_total = sum_b ceil(rows_b/256) * P_b.  results:
 * HOST array of n_inst.                                                    */
int qes_batch_sr_workspace_bytes(int dtype, int n_inst, int64_t n_params_total, int64_t n_samples_total,
                                 int64_t sr_part_total, size_t* bytes);
int qes_batch_sr_solve_cg(int dtype, int n_inst, const qes_batch_instance* inst, int n_ov_items,
                          const int32_t* ov_items, int n_ohu_items, const int32_t* ohu_items,
                          int64_t n_params_total, int64_t n_samples_total, int64_t sr_part_total,
                          const uint32_t* sample_bits, const void* tanh_theta, const void* eloc,
                          const qes_sr_options* opts, void* x_out, qes_sr_result* results,
                          void* workspace, size_t workspace_bytes, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* QES_B200_H */
