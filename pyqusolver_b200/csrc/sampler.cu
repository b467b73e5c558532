// Persistent Metropolis sampler: one warp per chain.
//
// Chain state: packed spins in shared memory; theta and tanh(theta) of the
// chain live in registers, lane l owning hidden units m = l + 32 r (r < MPL).
// A proposal costs one Philox call, O(M/32) complex FMAs per lane against the
// move's cosh/sinh table row, a per-lane log and one warp sum -- the
// reference instead re-evaluates the whole network for every exchange
// proposal (vmc.py:1050-1054).  An accepted move updates theta by the rank-1
// (flip) or rank-2 (exchange) column of W; theta is recomputed from the spins
// every `recompute_every` proposals to bound float32 drift.
//
// Reference semantics kept (vmc.py:1016-1097, spin_jax.py:51-158):
//   log_acc = min(beta*mu*Re dlogpsi, 0); accept iff log u < log_acc;
//   exchange with an invalid slot or equal spins is a no-op with dlogpsi = 0,
//   accepted (u < 1); proposed += 1 and accepted += keep for every proposal.
#include <algorithm>
#include <atomic>

#include "common.cuh"

#define QES_ARG_CHECK(cond, msg) do { if (!(cond)) { qes_set_last_message(msg); return QES_ERR_ARG; } } while (0)

constexpr int SMP_WARPS = 4;        // chains per block
constexpr int SMP_MAX_WORDS = 64;   // ns <= 2048

template <class T>
QES_D float log_abs(T v);
template <>
QES_D float log_abs<float>(float v) { return logf(fabsf(v)); }
template <>
QES_D float log_abs<float2>(float2 v) { return 0.5f * logf(v.x * v.x + v.y * v.y); }

// tanh(theta) for the acceptance cache, from the hardware exponential, sine/cosine and reciprocal
// approximations: a handful of instructions against the accurate library forms, whose cost
// dominated the accepted-move update (most proposals are accepted near initialisation).  The cache
// enters the ratio only as C + g t S, so an absolute error of a few 1e-7 in t moves the acceptance
// ratio by a relative ~1e-7, the size of its own float32 rounding; theta itself stays exact (it
// feeds log psi) and the forward, local-energy and SR kernels keep the accurate tanh.
//
// Real: tanh x = 1 - 2 / (e^{2x} + 1).  The divisor is at least one, so the absolute error stays
// below about 5e-7; e^{2x} overflows to +inf or underflows to 0 and gives exactly +-1, never NaN.
QES_D float tanh_cache(float x) { return 1.f - __fdividef(2.f, __expf(2.f * x) + 1.f); }
// Complex: the pole-safe form of tanhx, tanh(x+iy) = [sign(x)(1 - q^2) + i 4 q sin y cos y] /
// [(1 - q)^2 + 4 q cos^2 y] with q = e^{-2|x|} in (0, 1], so no term cancels except near the poles
// (x = 0, cos y = 0) where t is large in any evaluation; at an exact pole (den = 0 in float32) the
// divisor is clamped to 1e-30 so that the cache holds a finite value instead of 0/0 = NaN (a NaN
// would silently decide every later acceptance of the chain).  y is first reduced to [-pi, pi] by
// Cody-Waite reduction (2 pi split into a float head and tail) because the hardware sine/cosine
// is accurate (abs error ~4e-7) only on that interval.
QES_D float2 tanh_cache(float2 z) {
  const float q = __expf(-2.f * fabsf(z.x));
  const float em = q - 1.f;                                      // q - 1, exact subtraction
  const float k = rintf(z.y * 0.15915494309189535f);             // y / (2 pi), nearest integer
  float y = fmaf(-k, 6.28318548202514648f, z.y);                 // float(2 pi)
  y = fmaf(-k, -1.7484555314695172e-7f, y);                      // 2 pi - float(2 pi)
  float sy, cy;
  __sincosf(y, &sy, &cy);
  const float den = fmaxf(em * em + 4.f * q * cy * cy, 1e-30f);
  const float re = __fdividef(copysignf(-em * (2.f + em), z.x), den);
  const float im = __fdividef(4.f * q * sy * cy, den);
  return make_float2(re, im);
}

// theta / tanh(theta) of one chain: lane l owns hidden units m = l + 32 r (r < MPL), held in
// registers (narrow caches) or in a per-warp slice of shared memory (wide caches, where a
// register-resident cache would cap the SM at a few warps)
template <class T, int MPL, bool SMEM>
struct ThetaCache;
template <class T, int MPL>
struct ThetaCache<T, MPL, false> {
  static constexpr int kMPL = MPL;
  static constexpr bool kSmem = false;
  T th_[MPL], tn_[MPL];
  QES_D void bind(T*, int, int) {}
  QES_D T& th(int r) { return th_[r]; }
  QES_D T& tn(int r) { return tn_[r]; }
};
template <class T, int MPL>
struct ThetaCache<T, MPL, true> {
  static constexpr int kMPL = MPL;
  static constexpr bool kSmem = true;
  T* th_;
  T* tn_;
  // the warp's slice holds rows = ceil(nh / 32) rows of theta, then as many of tanh(theta); rows at
  // or past `rows` do not exist and are never touched
  QES_D void bind(T* warp_slice, int lane, int rows) { th_ = warp_slice + lane; tn_ = warp_slice + 32 * rows + lane; }
  QES_D T& th(int r) { return th_[32 * r]; }
  QES_D T& tn(int r) { return tn_[32 * r]; }
};

// lane: the thread's index within its chain (warp lane, or warp-in-chain * 32 + lane when KW warps
// share a chain); unit m = lane + 32 KW r
template <class T, class Cache, int KW = 1>
QES_D void full_theta(int ns, int nh, int lane, const uint32_t* cfg, const T* __restrict__ b,
                      const T* __restrict__ W, Cache& c) {
  constexpr int MPL = Cache::kMPL;
  constexpr int STRIDE = 32 * KW;
  // accumulate CH units per lane in registers, then store (CH = MPL for register caches)
  constexpr int CH = Cache::kSmem ? 16 : MPL;
#pragma unroll
  for (int c0 = 0; c0 < MPL; c0 += CH) {
    T acc[CH];
#pragma unroll
    for (int r = 0; r < CH; ++r) {
      const int m = lane + STRIDE * (c0 + r);
      acc[r] = (m < nh) ? b[m] : ScalarTraits<T>::zero();
    }
    auto site = [&](int i) {
      const float sg = ((cfg[i >> 5] >> (i & 31)) & 1u) ? 1.f : -1.f;
      const T* wr = W + (int64_t)i * nh;
#pragma unroll
      for (int r = 0; r < CH; ++r) {
        const int m = lane + STRIDE * (c0 + r);
        if (m < nh) acc[r] = addx(acc[r], scal(sg, wr[m]));
      }
    };
    if constexpr (CH >= 16) {
#pragma unroll 4
      for (int i = 0; i < ns; ++i) site(i);
    } else {
      for (int i = 0; i < ns; ++i) site(i);
    }
#pragma unroll
    for (int r = 0; r < CH; ++r) {
      if (!Cache::kSmem || 32 * (c0 + r) < nh) {
        c.th(c0 + r) = acc[r];
        c.tn(c0 + r) = tanh_cache(acc[r]);
      }
    }
  }
}

// red (KW > 1): KW shared slots for the sum over the chain's warps (block-wide barriers)
template <class T, class Cache, int KW = 1>
QES_D T chain_logpsi(int ns, int nh, int lane, const uint32_t* cfg, const T* __restrict__ a, Cache& c,
                     T* red = nullptr) {
  constexpr int MPL = Cache::kMPL;
  constexpr int STRIDE = 32 * KW;
  T s = ScalarTraits<T>::zero();
#pragma unroll
  for (int r = 0; r < MPL; ++r) {
    const int m = lane + STRIDE * r;
    if (m < nh) s = addx(s, log_cosh(c.th(r)));
  }
  for (int i = lane; i < ns; i += STRIDE) {
    const float sg = ((cfg[i >> 5] >> (i & 31)) & 1u) ? 1.f : -1.f;
    s = addx(s, scal(sg, a[i]));
  }
  s = warp_sum(s);
  if constexpr (KW > 1) {
    if ((lane & 31) == 0) red[lane >> 5] = s;
    __syncthreads();
    s = red[0];
    for (int w = 1; w < KW; ++w) s = addx(s, red[w]);
    __syncthreads();                                  // the slots are reused by the next call
  }
  return s;
}

// barrier over the threads of one chain: its warp, or its block when KW warps share the chain
template <int KW>
QES_D void chain_sync() {
  if constexpr (KW == 1) __syncwarp();
  else __syncthreads();
}

// Everything one chain needs; pointers are already offset to the chain's problem.
template <class T>
struct ChainCtx {
  int ns, nh, n_chains, deg, sweep_steps, recompute_every, num_samples;
  int64_t therm_steps_total;
  float beta_mu;
  uint32_t k0, k1;
  int64_t chain_id;                         // global chain id (Philox counter word 0)
  const T *a, *b, *W, *flipC, *flipS, *pairC, *pairS;
  const int32_t *nbr, *nbr_pair, *pair_i, *pair_j;
};

// Runs proposals for chain `chain` (index within its problem) with the
// problem's packed spins staged in `cw` (shared memory, one warp).
// KW > 1: the chain runs on a whole block of KW warps (register caches only); thread gl = threadIdx.x
// owns units gl + 32 KW r, the block draws the Philox numbers of 32 KW proposals at once into `rng`
// (shared memory), every thread takes the same decision, and the log-ratio is summed over the warps through `red_la` (two sets of KW slots, used
// alternately) and `red_lp` (KW slots) in shared memory, in warp order.
template <class T, int MPL, int RULE, bool SMEM = false, int KW = 1>
QES_D void run_chain(const ChainCtx<T>& P, int chain, uint32_t* cw, T* theta_slice, uint32_t* __restrict__ chain_bits,
                     uint64_t* __restrict__ chain_step, int32_t* __restrict__ proposed,
                     int32_t* __restrict__ accepted, uint32_t* __restrict__ sample_bits,
                     T* __restrict__ sample_logpsi, T* __restrict__ last_logpsi, float* red_la = nullptr,
                     T* red_lp = nullptr, uint4* rng = nullptr) {
  static_assert(KW == 1 || !SMEM, "chains shared by several warps keep their caches in registers");
  constexpr int STRIDE = 32 * KW;
  const int lane = KW == 1 ? (int)(threadIdx.x & 31) : (int)threadIdx.x;   // index within the chain
  const int ns = P.ns, nh = P.nh, nw = n_words(ns);
  const T* __restrict__ a = P.a;
  const T* __restrict__ b = P.b;
  const T* __restrict__ W = P.W;
  for (int q = lane; q < nw; q += STRIDE) cw[q] = chain_bits[(int64_t)chain * nw + q];
  chain_sync<KW>();
  int red_par = 0;

  const uint32_t cid = (uint32_t)P.chain_id;
  uint64_t step = chain_step[chain];
  int32_t n_prop = proposed[chain], n_acc = accepted[chain];
  const int recompute = P.recompute_every > 0 ? P.recompute_every : ns;
  const float bm = P.beta_mu;

  ThetaCache<T, MPL, SMEM> cache;
  cache.bind(theta_slice, lane, (nh + 31) >> 5);
  full_theta<T, ThetaCache<T, MPL, SMEM>, KW>(ns, nh, lane, cw, b, W, cache);
  int since = 0;

  const int64_t total = P.therm_steps_total + (int64_t)P.num_samples * P.sweep_steps;
  int64_t rec = 0;
  int64_t next_record = P.therm_steps_total + P.sweep_steps;

  // The Philox draws of STRIDE consecutive proposals are computed at once, thread q taking step + q
  // (one counter-mode call per STRIDE proposals instead of one per proposal in every thread; the same
  // numbers, so the same chain): one-warp chains hand them out by shuffles (heis10x10 sampling
  // 1.47 -> 1.28 ms), multi-warp chains through `rng` in shared memory (three more live registers
  // per thread pushed their kernel past its register cap).
  uint32_t pb_x = 0, pb_y = 0;
  float pb_lu = 0.f;
  int pb_k = STRIDE;
  for (int64_t it = 0; it < total; ++it) {
    Philox4 r;
    float log_u;
    if constexpr (KW == 1) {
      if (pb_k == 32) {
        const uint64_t sb = step + (uint64_t)(threadIdx.x & 31);
        const Philox4 rb = philox4x32_10(cid, (uint32_t)sb, (uint32_t)(sb >> 32), QES_STREAM_PROPOSAL, P.k0, P.k1);
        pb_x = rb.x;
        pb_y = rb.y;
        pb_lu = logf(uniform_open(rb.z));
        pb_k = 0;
      }
      r.x = __shfl_sync(0xffffffffu, pb_x, pb_k);
      r.y = __shfl_sync(0xffffffffu, pb_y, pb_k);
      log_u = __shfl_sync(0xffffffffu, pb_lu, pb_k);
      ++pb_k;
    } else {
      if (pb_k == STRIDE) {
        chain_sync<KW>();                     // every thread has read the previous batch
        const uint64_t sb = step + (uint64_t)lane;
        const Philox4 rb = philox4x32_10(cid, (uint32_t)sb, (uint32_t)(sb >> 32), QES_STREAM_PROPOSAL, P.k0, P.k1);
        rng[lane] = make_uint4(rb.x, rb.y, __float_as_uint(logf(uniform_open(rb.z))), 0u);
        chain_sync<KW>();
        pb_k = 0;
      }
      const uint4 q = rng[pb_k++];
      r.x = q.x;
      r.y = q.y;
      log_u = __uint_as_float(q.z);
    }
    const int i = (int)bounded_u32(r.x, (uint32_t)ns);
    bool moved;
    int i0 = i, j0 = -1;        // sites flipped (j0 = -1 for a single flip)
    const T* Crow;
    const T* Srow;
    if (RULE == QES_RULE_LOCAL) {
      moved = true;
      Crow = P.flipC + (int64_t)i * nh;
      Srow = P.flipS + (int64_t)i * nh;
    } else {
      const int kk = (int)bounded_u32(r.y, (uint32_t)P.deg);
      const int j = P.nbr[i * P.deg + kk];
      moved = false;
      Crow = P.flipC; Srow = P.flipS;
      if (j >= 0) {
        const uint32_t bi = (cw[i >> 5] >> (i & 31)) & 1u;
        const uint32_t bj = (cw[j >> 5] >> (j & 31)) & 1u;
        if (bi != bj) {
          const int p = P.nbr_pair[i * P.deg + kk];
          moved = true;
          i0 = P.pair_i[p]; j0 = P.pair_j[p];
          Crow = P.pairC + (int64_t)p * nh;
          Srow = P.pairS + (int64_t)p * nh;
        }
      }
    }
    float re_delta = 0.f;
    float g = 0.f;
    if (moved) {
      g = ((cw[i0 >> 5] >> (i0 & 31)) & 1u) ? -1.f : 1.f;      // -sigma_i0
      T prod = ScalarTraits<T>::one();
      int ex = 0;
      if constexpr (MPL >= 16) {
        // the table row is fetched a chunk ahead of the product so that its L2 round trips overlap;
        // units beyond nh read as (C, S) = (1, 0), an exact factor of one
        // 12 units per chunk for real shared-memory caches (measured faster than 8 or 16 on nh = 1600:
        // fewer registers live at 128); chunks past MPL read as factors of one
        constexpr int PF = (SMEM && !ScalarTraits<T>::is_complex) ? 12 : 16;
        T cb[2][PF], sb[2][PF];
#pragma unroll
        for (int q = 0; q < PF; ++q) {
          const int m = lane + STRIDE * q;
          cb[0][q] = (m < nh) ? Crow[m] : ScalarTraits<T>::one();
          sb[0][q] = (m < nh) ? Srow[m] : ScalarTraits<T>::zero();
        }
#pragma unroll
        for (int c0 = 0; c0 < MPL; c0 += PF) {
          const int cur = (c0 / PF) & 1;
          if (c0 + PF < MPL) {
#pragma unroll
            for (int q = 0; q < PF; ++q) {
              const int m = lane + STRIDE * (c0 + PF + q);
              cb[cur ^ 1][q] = (m < nh) ? Crow[m] : ScalarTraits<T>::one();
              sb[cur ^ 1][q] = (m < nh) ? Srow[m] : ScalarTraits<T>::zero();
            }
          }
#pragma unroll
          for (int q = 0; q < PF; ++q) {
            const int rr = c0 + q;
            const T t = (!SMEM || STRIDE * rr < nh) ? cache.tn(rr) : ScalarTraits<T>::zero();
            prod = mulx(prod, ratio_factor(cb[cur][q], g, t, sb[cur][q]));
            if ((rr & 7) == 7) renorm(prod, ex);
          }
        }
      } else {
#pragma unroll
        for (int rr = 0; rr < MPL; ++rr) {
          const int m = lane + STRIDE * rr;
          if (m < nh) prod = mulx(prod, ratio_factor(Crow[m], g, cache.tn(rr), Srow[m]));
          if ((rr & 7) == 7) renorm(prod, ex);
        }
      }
      float la = log_abs<T>(prod) + 0.69314718055994531f * (float)ex;
      la = warp_sum(la);
      if constexpr (KW > 1) {
        // every reduction is separated from the one two before it by the barrier of the one between,
        // so alternating slot sets cannot be overwritten while a warp still reads them
        float* slots = red_la + red_par * KW;
        if ((lane & 31) == 0) slots[lane >> 5] = la;
        __syncthreads();
        la = slots[0];
        for (int w = 1; w < KW; ++w) la += slots[w];
        red_par ^= 1;
      }
      T av = a[i0];
      if (j0 >= 0) av = addx(av, scal(-1.f, a[j0]));
      re_delta = la + 2.f * g * to_re(av);
    }
    const float log_acc = fminf(bm * re_delta, 0.f);
    const bool keep = log_u < log_acc;
    if (keep && moved) {
      const T* wi = W + (int64_t)i0 * nh;
      const T* wj = W + (int64_t)(j0 >= 0 ? j0 : i0) * nh;
      if constexpr (MPL >= 16) {
        constexpr int PU = 16;
#pragma unroll
        for (int c0 = 0; c0 < MPL; c0 += PU) {
          T d[PU];
#pragma unroll
          for (int q = 0; q < PU; ++q) {          // all loads of the chunk first
            const int m = lane + STRIDE * (c0 + q);
            d[q] = (m < nh) ? wi[m] : ScalarTraits<T>::zero();
            if (j0 >= 0) d[q] = addx(d[q], scal(-1.f, (m < nh) ? wj[m] : ScalarTraits<T>::zero()));
          }
#pragma unroll
          for (int q = 0; q < PU; ++q) {
            const int rr = c0 + q;
            if (lane + STRIDE * rr < nh) {
              const T t2 = addx(cache.th(rr), scal(2.f * g, d[q]));
              cache.th(rr) = t2;
              cache.tn(rr) = tanh_cache(t2);
            }
          }
        }
      } else {
#pragma unroll
        for (int rr = 0; rr < MPL; ++rr) {
          const int m = lane + STRIDE * rr;
          if (m < nh) {
            T d = wi[m];
            if (j0 >= 0) d = addx(d, scal(-1.f, wj[m]));
            const T t2 = addx(cache.th(rr), scal(2.f * g, d));
            cache.th(rr) = t2;
            cache.tn(rr) = tanh_cache(t2);
          }
        }
      }
      chain_sync<KW>();
      if (lane == 0) {
        cw[i0 >> 5] ^= 1u << (i0 & 31);
        if (j0 >= 0) cw[j0 >> 5] ^= 1u << (j0 & 31);
      }
      chain_sync<KW>();
    }
    n_prop += 1;
    n_acc += keep ? 1 : 0;
    ++step;
    if (++since >= recompute) {
      full_theta<T, ThetaCache<T, MPL, SMEM>, KW>(ns, nh, lane, cw, b, W, cache);
      since = 0;
    }
    if (it + 1 == next_record) {
      const int64_t row = rec * P.n_chains + chain;
      for (int q = lane; q < nw; q += STRIDE) sample_bits[row * nw + q] = cw[q];
      const T lp = chain_logpsi<T, ThetaCache<T, MPL, SMEM>, KW>(ns, nh, lane, cw, a, cache, red_lp);
      if (lane == 0 && sample_logpsi) sample_logpsi[row] = lp;
      ++rec;
      next_record += P.sweep_steps;
    }
  }
  for (int q = lane; q < nw; q += STRIDE) chain_bits[(int64_t)chain * nw + q] = cw[q];
  const T lp = chain_logpsi<T, ThetaCache<T, MPL, SMEM>, KW>(ns, nh, lane, cw, a, cache, red_lp);
  if (lane == 0) {
    chain_step[chain] = step;
    proposed[chain] = n_prop;
    accepted[chain] = n_acc;
    if (last_logpsi) last_logpsi[chain] = lp;
  }
  chain_sync<KW>();
}

// Wide theta caches (SMEM = true) live in dynamic shared memory, 2 * 32 * MPL elements per warp.
// MINB > 1 caps the registers so that MINB blocks share an SM (more chains resident at once).
template <class T, int MPL, int RULE, bool SMEM, int MINB = 1>
__global__ void __launch_bounds__(32 * SMP_WARPS, MINB) sampler_kernel(
    qes_sampler_config cfg, const T* __restrict__ a, const T* __restrict__ b, const T* __restrict__ W,
    const T* __restrict__ flipC, const T* __restrict__ flipS, const int32_t* __restrict__ nbr,
    const int32_t* __restrict__ nbr_pair, const int32_t* __restrict__ pair_i, const int32_t* __restrict__ pair_j,
    const T* __restrict__ pairC, const T* __restrict__ pairS, uint32_t* __restrict__ chain_bits,
    uint64_t* __restrict__ chain_step, int32_t* __restrict__ proposed, int32_t* __restrict__ accepted,
    uint32_t* __restrict__ sample_bits, T* __restrict__ sample_logpsi, T* __restrict__ last_logpsi,
    const float* __restrict__ chain_beta) {
  __shared__ uint32_t cfg_sm[SMP_WARPS][SMP_MAX_WORDS];
  extern __shared__ __align__(16) uint8_t theta_sm[];
  const int wid = threadIdx.x >> 5;
  const int chain = blockIdx.x * SMP_WARPS + wid;
  if (chain >= cfg.n_chains) return;            // whole warp leaves together
  ChainCtx<T> P;
  P.ns = cfg.ns; P.nh = cfg.nh; P.n_chains = cfg.n_chains; P.deg = cfg.deg; P.sweep_steps = cfg.sweep_steps;
  P.recompute_every = cfg.recompute_every; P.num_samples = cfg.num_samples;
  P.therm_steps_total = cfg.therm_steps_total;
  P.beta_mu = (chain_beta ? chain_beta[chain] : cfg.beta) * cfg.mu;     // per-chain beta: replica slots
  P.k0 = (uint32_t)(cfg.seed & 0xffffffffu); P.k1 = (uint32_t)(cfg.seed >> 32);
  P.chain_id = cfg.chain_offset + chain;
  P.a = a; P.b = b; P.W = W; P.flipC = flipC; P.flipS = flipS; P.pairC = pairC; P.pairS = pairS;
  P.nbr = nbr; P.nbr_pair = nbr_pair; P.pair_i = pair_i; P.pair_j = pair_j;
  T* slice = SMEM ? reinterpret_cast<T*>(theta_sm) + (size_t)wid * 2 * 32 * ((cfg.nh + 31) >> 5) : nullptr;
  run_chain<T, MPL, RULE, SMEM>(P, chain, cfg_sm[wid], slice, chain_bits, chain_step, proposed, accepted,
                                sample_bits, sample_logpsi, last_logpsi);
}

// Wide hidden layers, one chain per block of KW warps: every thread holds MPL units of the chain's
// theta / tanh cache in registers, so one proposal's table row is in flight at once (one L2 round
// trip) instead of being walked one chunk per round trip by a single warp, and no shared-memory cache
// caps the resident chains.  Same arithmetic per unit as the one-warp kernels; the log-ratio is summed
// per warp and then over the warps in order.  Four-warp chains are held to 72 registers (seven
// chains per SM): with the Philox draws batched the compiler took 96 (five chains per SM) and the
// 20x20 TFIM sampling ran 30.2 ms, capped 25.8 ms (28.7 ms before the batching; caps of 8 and 9
// chains per SM ran 29.0 and 27.0 ms).
template <class T, int MPL, int RULE, int KW>
__global__ void __launch_bounds__(32 * KW, KW == 4 ? 7 : 1) sampler_wide_kernel(
    qes_sampler_config cfg, const T* __restrict__ a, const T* __restrict__ b, const T* __restrict__ W,
    const T* __restrict__ flipC, const T* __restrict__ flipS, const int32_t* __restrict__ nbr,
    const int32_t* __restrict__ nbr_pair, const int32_t* __restrict__ pair_i, const int32_t* __restrict__ pair_j,
    const T* __restrict__ pairC, const T* __restrict__ pairS, uint32_t* __restrict__ chain_bits,
    uint64_t* __restrict__ chain_step, int32_t* __restrict__ proposed, int32_t* __restrict__ accepted,
    uint32_t* __restrict__ sample_bits, T* __restrict__ sample_logpsi, T* __restrict__ last_logpsi,
    const float* __restrict__ chain_beta) {
  __shared__ uint32_t cw[SMP_MAX_WORDS];
  __shared__ float red_la[2 * KW];
  __shared__ T red_lp[KW];
  __shared__ uint4 rng[32 * KW];
  const int chain = blockIdx.x;                 // the grid is exactly n_chains blocks
  ChainCtx<T> P;
  P.ns = cfg.ns; P.nh = cfg.nh; P.n_chains = cfg.n_chains; P.deg = cfg.deg; P.sweep_steps = cfg.sweep_steps;
  P.recompute_every = cfg.recompute_every; P.num_samples = cfg.num_samples;
  P.therm_steps_total = cfg.therm_steps_total;
  P.beta_mu = (chain_beta ? chain_beta[chain] : cfg.beta) * cfg.mu;
  P.k0 = (uint32_t)(cfg.seed & 0xffffffffu); P.k1 = (uint32_t)(cfg.seed >> 32);
  P.chain_id = cfg.chain_offset + chain;
  P.a = a; P.b = b; P.W = W; P.flipC = flipC; P.flipS = flipS; P.pairC = pairC; P.pairS = pairS;
  P.nbr = nbr; P.nbr_pair = nbr_pair; P.pair_i = pair_i; P.pair_j = pair_j;
  run_chain<T, MPL, RULE, false, KW>(P, chain, cw, nullptr, chain_bits, chain_step, proposed, accepted, sample_bits,
                                     sample_logpsi, last_logpsi, red_la, red_lp, rng);
}

// register caches up to 16 units per lane (real) / 8 (complex); wider ones in shared memory
template <class T, int MPL>
constexpr bool sampler_smem_cache() { return MPL > (ScalarTraits<T>::is_complex ? 8 : 16); }

// wide layers: chains of KW warps (1), or one warp per chain with a shared-memory cache (0)
static std::atomic<int> g_smp_wide{1};
extern "C" int qes_sampler_set_wide(int on) {
  g_smp_wide.store(on ? 1 : 0);
  return QES_OK;
}

template <class T, int MPL, int KW>
static int launch_sampler_wide(const qes_sampler_config* cfg, const void* a, const void* b, const void* W,
                               const void* flipC, const void* flipS, const int32_t* nbr, const int32_t* nbr_pair,
                               const int32_t* pi, const int32_t* pj, const void* pairC, const void* pairS,
                               uint32_t* chain_bits, uint64_t* chain_step, int32_t* proposed, int32_t* accepted,
                               uint32_t* sample_bits, void* sample_logpsi, void* last_logpsi, const float* chain_beta,
                               cudaStream_t st) {
#define QES_SMPW_ARGS                                                                                             \
  *cfg, (const T*)a, (const T*)b, (const T*)W, (const T*)flipC, (const T*)flipS, nbr, nbr_pair, pi, pj,            \
      (const T*)pairC, (const T*)pairS, chain_bits, chain_step, proposed, accepted, sample_bits, (T*)sample_logpsi, \
      (T*)last_logpsi, chain_beta
  if (cfg->rule == QES_RULE_LOCAL)
    sampler_wide_kernel<T, MPL, QES_RULE_LOCAL, KW><<<(unsigned)cfg->n_chains, 32 * KW, 0, st>>>(QES_SMPW_ARGS);
  else
    sampler_wide_kernel<T, MPL, QES_RULE_EXCHANGE, KW><<<(unsigned)cfg->n_chains, 32 * KW, 0, st>>>(QES_SMPW_ARGS);
#undef QES_SMPW_ARGS
  QES_LAUNCH_CHECK();
  return QES_OK;
}

template <class T, int MPL, int RULE, bool SM, int MINB>
static int launch_sampler_kernel(unsigned grid, size_t smem, const qes_sampler_config* cfg, const void* a,
                                 const void* b, const void* W, const void* flipC, const void* flipS,
                                 const int32_t* nbr, const int32_t* nbr_pair, const int32_t* pi, const int32_t* pj,
                                 const void* pairC, const void* pairS, uint32_t* chain_bits, uint64_t* chain_step,
                                 int32_t* proposed, int32_t* accepted, uint32_t* sample_bits, void* sample_logpsi,
                                 void* last_logpsi, const float* chain_beta, cudaStream_t st) {
  if (SM)
    QES_CUDA_CHECK(cudaFuncSetAttribute(sampler_kernel<T, MPL, RULE, SM, MINB>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  sampler_kernel<T, MPL, RULE, SM, MINB><<<grid, 32 * SMP_WARPS, smem, st>>>(
      *cfg, (const T*)a, (const T*)b, (const T*)W, (const T*)flipC, (const T*)flipS, nbr, nbr_pair, pi, pj,
      (const T*)pairC, (const T*)pairS, chain_bits, chain_step, proposed, accepted, sample_bits,
      (T*)sample_logpsi, (T*)last_logpsi, chain_beta);
  QES_LAUNCH_CHECK();
  return QES_OK;
}

// Register-resident caches: the kernel with the register cap (7 blocks of 4 chains per SM) runs
// when it needs fewer waves of resident chains than the uncapped one (more chains than one wave
// of the latter) and spills no more than it; otherwise the uncapped kernel.  Both run the same
// arithmetic in the same order, so the choice never changes a sample.
// qes_sampler_set_capped: 0 never, 1 by the wave count (default), 2 always where instantiated.
constexpr int SMP_CAPPED_BLOCKS = 7;
// Shared-memory caches (wide hidden layers): capped at 128 registers so that four blocks (16
// chains) share an SM where their slices fit; uncapped, up to 255 registers left two.
constexpr int SMP_SMEM_BLOCKS = 4;
static std::atomic<int> g_smp_capped{1};
extern "C" int qes_sampler_set_capped(int mode) {
  if (mode < 0 || mode > 2) {
    qes_set_last_message("qes_sampler_set_capped: mode must be 0, 1 or 2");
    return QES_ERR_ARG;
  }
  g_smp_capped.store(mode);
  return QES_OK;
}

template <class T, int MPL, int RULE>
static int sampler_pick_capped(const qes_sampler_config* cfg, bool* capped) {
  *capped = false;
  const int mode = g_smp_capped.load(std::memory_order_relaxed);
  if (mode == 0) return QES_OK;
  if (mode == 2) {
    *capped = true;
    return QES_OK;
  }
  cudaFuncAttributes f1{}, f7{};
  QES_CUDA_CHECK(cudaFuncGetAttributes(&f1, sampler_kernel<T, MPL, RULE, false, 1>));
  QES_CUDA_CHECK(cudaFuncGetAttributes(&f7, sampler_kernel<T, MPL, RULE, false, SMP_CAPPED_BLOCKS>));
  if (f7.localSizeBytes > f1.localSizeBytes) return QES_OK;
  int dev = 0, nsm = 0, b1 = 0, b7 = 0;
  QES_CUDA_CHECK(cudaGetDevice(&dev));
  QES_CUDA_CHECK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  QES_CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b1, sampler_kernel<T, MPL, RULE, false, 1>,
                                                               32 * SMP_WARPS, 0));
  QES_CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
      &b7, sampler_kernel<T, MPL, RULE, false, SMP_CAPPED_BLOCKS>, 32 * SMP_WARPS, 0));
  const int64_t n = cfg->n_chains;
  const int64_t cap1 = (int64_t)std::max(b1, 1) * SMP_WARPS * nsm, cap7 = (int64_t)std::max(b7, 1) * SMP_WARPS * nsm;
  *capped = (n + cap7 - 1) / cap7 < (n + cap1 - 1) / cap1;
  return QES_OK;
}

template <class T, int MPL>
static int launch_sampler_mpl(const qes_sampler_config* cfg, const void* a, const void* b, const void* W,
                              const void* flipC, const void* flipS, const int32_t* nbr, const int32_t* nbr_pair,
                              const int32_t* pi, const int32_t* pj, const void* pairC, const void* pairS,
                              uint32_t* chain_bits, uint64_t* chain_step, int32_t* proposed, int32_t* accepted,
                              uint32_t* sample_bits, void* sample_logpsi, void* last_logpsi, const float* chain_beta,
                              cudaStream_t st) {
  constexpr bool SM = sampler_smem_cache<T, MPL>();
  const unsigned grid = (unsigned)((cfg->n_chains + SMP_WARPS - 1) / SMP_WARPS);
  // shared-memory caches are sized to the hidden layer (ceil(nh / 32) rows), not to MPL
  const size_t smem = SM ? (size_t)SMP_WARPS * 2 * 32 * ((cfg->nh + 31) / 32) * sizeof(T) : 0;
#define QES_SMP_ARGS grid, smem, cfg, a, b, W, flipC, flipS, nbr, nbr_pair, pi, pj, pairC, pairS, chain_bits, \
                     chain_step, proposed, accepted, sample_bits, sample_logpsi, last_logpsi, chain_beta, st
  if (cfg->rule == QES_RULE_LOCAL) {
    if constexpr (!SM) {
      bool capped = false;
      if (int rc = sampler_pick_capped<T, MPL, QES_RULE_LOCAL>(cfg, &capped)) return rc;
      if (capped) return launch_sampler_kernel<T, MPL, QES_RULE_LOCAL, false, SMP_CAPPED_BLOCKS>(QES_SMP_ARGS);
    }
    return launch_sampler_kernel<T, MPL, QES_RULE_LOCAL, SM, SM ? SMP_SMEM_BLOCKS : 1>(QES_SMP_ARGS);
  }
  if constexpr (!SM) {
    bool capped = false;
    if (int rc = sampler_pick_capped<T, MPL, QES_RULE_EXCHANGE>(cfg, &capped)) return rc;
    if (capped) return launch_sampler_kernel<T, MPL, QES_RULE_EXCHANGE, false, SMP_CAPPED_BLOCKS>(QES_SMP_ARGS);
  }
  return launch_sampler_kernel<T, MPL, QES_RULE_EXCHANGE, SM, SM ? SMP_SMEM_BLOCKS : 1>(QES_SMP_ARGS);
#undef QES_SMP_ARGS
}

template <class T>
static int launch_sampler(int mpl_needed, int mpl_max, const qes_sampler_config* cfg, const void* a, const void* b,
                          const void* W, const void* flipC, const void* flipS, const int32_t* nbr,
                          const int32_t* nbr_pair, const int32_t* pi, const int32_t* pj, const void* pairC,
                          const void* pairS, uint32_t* chain_bits, uint64_t* chain_step, int32_t* proposed,
                          int32_t* accepted, uint32_t* sample_bits, void* sample_logpsi, void* last_logpsi,
                          const float* chain_beta, cudaStream_t st) {
#define QES_SMP_CASE(M)                                                                                          \
  if (mpl_needed <= M && M <= mpl_max)                                                                           \
    return launch_sampler_mpl<T, M>(cfg, a, b, W, flipC, flipS, nbr, nbr_pair, pi, pj, pairC, pairS, chain_bits, \
                                    chain_step, proposed, accepted, sample_bits, sample_logpsi, last_logpsi,      \
                                    chain_beta, st);
  QES_SMP_CASE(1)
  QES_SMP_CASE(2)
  QES_SMP_CASE(4)
  QES_SMP_CASE(8)
  QES_SMP_CASE(16)
  if constexpr (!ScalarTraits<T>::is_complex) {
    QES_SMP_CASE(32)
    QES_SMP_CASE(64)
  }
#undef QES_SMP_CASE
  qes_set_last_message("qes_sampler_run: too many hidden units for the register-resident theta cache");
  return QES_ERR_SIZE;
}

// Chains of several warps for hidden layers beyond one warp's register cache: KW = 2, 4 or 8 warps
// of MPL = 16 (real) / 8 (complex) units per thread.  Returns QES_ERR_SIZE when none fits.
template <class T>
static int launch_sampler_multiwarp(int mpl_needed, const qes_sampler_config* cfg, const void* a, const void* b,
                                    const void* W, const void* flipC, const void* flipS, const int32_t* nbr,
                                    const int32_t* nbr_pair, const int32_t* pi, const int32_t* pj,
                                    const void* pairC, const void* pairS, uint32_t* chain_bits,
                                    uint64_t* chain_step, int32_t* proposed, int32_t* accepted,
                                    uint32_t* sample_bits, void* sample_logpsi, void* last_logpsi,
                                    const float* chain_beta, cudaStream_t st) {
  constexpr int M = ScalarTraits<T>::is_complex ? 8 : 16;
#define QES_SMPW_CASE(K)                                                                                        \
  if (mpl_needed <= K * M)                                                                                      \
    return launch_sampler_wide<T, M, K>(cfg, a, b, W, flipC, flipS, nbr, nbr_pair, pi, pj, pairC, pairS,        \
                                        chain_bits, chain_step, proposed, accepted, sample_bits, sample_logpsi, \
                                        last_logpsi, chain_beta, st);
  QES_SMPW_CASE(2)
  QES_SMPW_CASE(4)
  QES_SMPW_CASE(8)
#undef QES_SMPW_CASE
  qes_set_last_message("qes_sampler_run: too many hidden units for the multi-warp chains");
  return QES_ERR_SIZE;
}

static int sampler_run_impl(int dtype, const qes_sampler_config* cfg, const float* chain_beta, const void* a,
                            const void* b, const void* W, const void* flipCt, const void* flipSt,
                            const int32_t* nbr_table, const int32_t* nbr_pair, const int32_t* pair_i,
                            const int32_t* pair_j, int n_pairs, const void* pairCt, const void* pairSt,
                            uint32_t* chain_bits, uint64_t* chain_step, int32_t* proposed, int32_t* accepted,
                            uint32_t* sample_bits, void* sample_logpsi, void* last_logpsi, void* stream) {
  QES_ARG_CHECK(cfg != nullptr, "qes_sampler_run: null config");
  QES_ARG_CHECK(dtype == QES_DTYPE_F32 || dtype == QES_DTYPE_C64, "qes_sampler_run: bad dtype");
  QES_ARG_CHECK(cfg->ns > 0 && cfg->nh > 0 && cfg->n_chains >= 0 && cfg->num_samples >= 0, "qes_sampler_run: bad sizes");
  QES_ARG_CHECK(cfg->therm_steps_total >= 0 && cfg->sweep_steps >= 1, "qes_sampler_run: bad schedule");
  QES_ARG_CHECK(n_words(cfg->ns) <= SMP_MAX_WORDS, "qes_sampler_run: ns > 2048");
  QES_ARG_CHECK(a && b && W && chain_bits && chain_step && proposed && accepted, "qes_sampler_run: null pointer");
  QES_ARG_CHECK(cfg->num_samples == 0 || sample_bits, "qes_sampler_run: null sample buffer");
  if (cfg->rule == QES_RULE_LOCAL) {
    QES_ARG_CHECK(flipCt && flipSt, "qes_sampler_run: LOCAL needs flip tables");
  } else if (cfg->rule == QES_RULE_EXCHANGE) {
    QES_ARG_CHECK(cfg->deg > 0 && nbr_table && nbr_pair && pair_i && pair_j && pairCt && pairSt && n_pairs > 0,
                  "qes_sampler_run: EXCHANGE needs neighbour and pair tables");
  } else {
    QES_ARG_CHECK(false, "qes_sampler_run: unknown rule");
  }
  if (cfg->n_chains == 0) return QES_OK;
  const int mpl = (cfg->nh + 31) / 32;
  cudaStream_t st = (cudaStream_t)stream;
  // hidden layers wider than one warp's register cache: chains of several warps (default), or one warp
  // per chain with the cache in shared memory (qes_sampler_set_wide(0))
  const int reg_max = dtype == QES_DTYPE_F32 ? 16 : 8;
  if (mpl > reg_max && g_smp_wide.load(std::memory_order_relaxed) != 0) {
    QES_ARG_CHECK(cfg->n_chains <= 0x7fffffff, "qes_sampler_run: too many chains");
    if (dtype == QES_DTYPE_F32)
      return launch_sampler_multiwarp<float>(mpl, cfg, a, b, W, flipCt, flipSt, nbr_table, nbr_pair, pair_i, pair_j,
                                             pairCt, pairSt, chain_bits, chain_step, proposed, accepted, sample_bits,
                                             sample_logpsi, last_logpsi, chain_beta, st);
    return launch_sampler_multiwarp<float2>(mpl, cfg, a, b, W, flipCt, flipSt, nbr_table, nbr_pair, pair_i, pair_j,
                                            pairCt, pairSt, chain_bits, chain_step, proposed, accepted, sample_bits,
                                            sample_logpsi, last_logpsi, chain_beta, st);
  }
  if (dtype == QES_DTYPE_F32)
    return launch_sampler<float>(mpl, 64, cfg, a, b, W, flipCt, flipSt, nbr_table, nbr_pair, pair_i, pair_j, pairCt,
                                 pairSt, chain_bits, chain_step, proposed, accepted, sample_bits, sample_logpsi,
                                 last_logpsi, chain_beta, st);
  return launch_sampler<float2>(mpl, 16, cfg, a, b, W, flipCt, flipSt, nbr_table, nbr_pair, pair_i, pair_j, pairCt,
                                pairSt, chain_bits, chain_step, proposed, accepted, sample_bits, sample_logpsi,
                                last_logpsi, chain_beta, st);
}

extern "C" int qes_sampler_run(int dtype, const qes_sampler_config* cfg, const void* a, const void* b,
                               const void* W, const void* flipCt, const void* flipSt, const int32_t* nbr_table,
                               const int32_t* nbr_pair, const int32_t* pair_i, const int32_t* pair_j, int n_pairs,
                               const void* pairCt, const void* pairSt, uint32_t* chain_bits, uint64_t* chain_step,
                               int32_t* proposed, int32_t* accepted, uint32_t* sample_bits, void* sample_logpsi,
                               void* last_logpsi, void* stream) {
  return sampler_run_impl(dtype, cfg, nullptr, a, b, W, flipCt, flipSt, nbr_table, nbr_pair, pair_i, pair_j, n_pairs,
                          pairCt, pairSt, chain_bits, chain_step, proposed, accepted, sample_bits, sample_logpsi,
                          last_logpsi, stream);
}

extern "C" int qes_sampler_run_betas(int dtype, const qes_sampler_config* cfg, const float* chain_beta,
                                     const void* a, const void* b, const void* W, const void* flipCt,
                                     const void* flipSt, const int32_t* nbr_table, const int32_t* nbr_pair,
                                     const int32_t* pair_i, const int32_t* pair_j, int n_pairs, const void* pairCt,
                                     const void* pairSt, uint32_t* chain_bits, uint64_t* chain_step,
                                     int32_t* proposed, int32_t* accepted, uint32_t* sample_bits,
                                     void* sample_logpsi, void* last_logpsi, void* stream) {
  QES_ARG_CHECK(chain_beta != nullptr, "qes_sampler_run_betas: null chain_beta");
  return sampler_run_impl(dtype, cfg, chain_beta, a, b, W, flipCt, flipSt, nbr_table, nbr_pair, pair_i, pair_j,
                          n_pairs, pairCt, pairSt, chain_bits, chain_step, proposed, accepted, sample_bits,
                          sample_logpsi, last_logpsi, stream);
}

// ----------------------------------------------------------------------------
// Parallel tempering: replica slots r = 0..R-1 of n_chains chains each (chain
// index r * n_chains + c) carry beta labels; after each round adjacent slots
// (r, r+1) with r % 2 == phase exchange labels per chain with probability
// min(1, exp((beta_r - beta_r+1) mu (Re log psi_r+1 - Re log psi_r))).
// The phase is one Philox draw per round (counter (round, 0, 0, 4)); the
// uniform of pair r in chain c is counter (c, round, r, 5).
// ----------------------------------------------------------------------------
constexpr uint32_t QES_STREAM_PT_PHASE = 4, QES_STREAM_PT_SWAP = 5;

template <class T>
__global__ void pt_swap_kernel(int R, int n_chains, const T* __restrict__ logpsi, float* __restrict__ beta, float mu,
                               uint32_t k0, uint32_t k1, int64_t round, int* __restrict__ swaps) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n_chains) return;
  const Philox4 ph = philox4x32_10((uint32_t)round, (uint32_t)(round >> 32), 0u, QES_STREAM_PT_PHASE, k0, k1);
  const int phase = (int)(ph.x & 1u);
  for (int r = phase; r + 1 < R; r += 2) {
    const float bi = beta[(int64_t)r * n_chains + c], bj = beta[(int64_t)(r + 1) * n_chains + c];
    const double li = (double)to_re(logpsi[(int64_t)r * n_chains + c]);
    const double lj = (double)to_re(logpsi[(int64_t)(r + 1) * n_chains + c]);
    const double log_acc = ((double)bi - (double)bj) * (double)mu * (lj - li);
    const Philox4 u = philox4x32_10((uint32_t)c, (uint32_t)round, (uint32_t)r, QES_STREAM_PT_SWAP, k0, k1);
    if (log((double)uniform_open(u.x)) < fmin(log_acc, 0.0)) {
      beta[(int64_t)r * n_chains + c] = bj;
      beta[(int64_t)(r + 1) * n_chains + c] = bi;
      if (swaps) atomicAdd(&swaps[r], 1);
    }
  }
}

// copies, for every chain c, the slot whose beta equals target (the physical sector) to record row c
template <class T>
__global__ void pt_collect_kernel(int R, int n_chains, int nw, const float* __restrict__ beta, float target,
                                  const uint32_t* __restrict__ chain_bits, const T* __restrict__ logpsi,
                                  uint32_t* __restrict__ out_bits, T* __restrict__ out_logpsi) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n_chains) return;
  int slot = 0;
  for (int r = R - 1; r >= 0; --r)
    if (fabsf(beta[(int64_t)r * n_chains + c] - target) < 1e-5f) slot = r;   // first match
  const int64_t src = (int64_t)slot * n_chains + c;
  for (int q = 0; q < nw; ++q) out_bits[(int64_t)c * nw + q] = chain_bits[src * nw + q];
  if (out_logpsi) out_logpsi[c] = logpsi[src];
}

template <class T>
__global__ void tanh_cache_kernel(int64_t n, const T* __restrict__ x, T* __restrict__ y) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) y[i] = tanh_cache(x[i]);
}

extern "C" int qes_sampler_tanh_cache(int dtype, int64_t n, const void* x, void* y, void* stream) {
  QES_ARG_CHECK(dtype == QES_DTYPE_F32 || dtype == QES_DTYPE_C64, "qes_sampler_tanh_cache: bad dtype");
  QES_ARG_CHECK(n >= 0, "qes_sampler_tanh_cache: bad size");
  if (n == 0) return QES_OK;
  QES_ARG_CHECK(x && y, "qes_sampler_tanh_cache: null pointer");
  const int bs = 256;
  const unsigned grid = (unsigned)((n + bs - 1) / bs);
  if (dtype == QES_DTYPE_F32)
    tanh_cache_kernel<float><<<grid, bs, 0, (cudaStream_t)stream>>>(n, (const float*)x, (float*)y);
  else
    tanh_cache_kernel<float2><<<grid, bs, 0, (cudaStream_t)stream>>>(n, (const float2*)x, (float2*)y);
  QES_LAUNCH_CHECK();
  return QES_OK;
}

extern "C" int qes_pt_swap(int dtype, int n_replicas, int n_chains, const void* logpsi, float* chain_beta, float mu,
                           uint64_t seed, int64_t round, int* swaps_accepted, void* stream) {
  QES_ARG_CHECK(dtype == QES_DTYPE_F32 || dtype == QES_DTYPE_C64, "qes_pt_swap: bad dtype");
  QES_ARG_CHECK(n_replicas >= 1 && n_chains >= 0 && round >= 0, "qes_pt_swap: bad sizes");
  if (n_chains == 0 || n_replicas < 2) return QES_OK;
  QES_ARG_CHECK(logpsi && chain_beta, "qes_pt_swap: null pointer");
  const int bs = 128;
  const uint32_t k0 = (uint32_t)(seed & 0xffffffffu), k1 = (uint32_t)(seed >> 32);
  if (dtype == QES_DTYPE_F32)
    pt_swap_kernel<float><<<(n_chains + bs - 1) / bs, bs, 0, (cudaStream_t)stream>>>(
        n_replicas, n_chains, (const float*)logpsi, chain_beta, mu, k0, k1, round, swaps_accepted);
  else
    pt_swap_kernel<float2><<<(n_chains + bs - 1) / bs, bs, 0, (cudaStream_t)stream>>>(
        n_replicas, n_chains, (const float2*)logpsi, chain_beta, mu, k0, k1, round, swaps_accepted);
  QES_LAUNCH_CHECK();
  return QES_OK;
}

extern "C" int qes_pt_collect(int dtype, int n_replicas, int n_chains, int ns, const float* chain_beta,
                              float target_beta, const uint32_t* chain_bits, const void* logpsi, uint32_t* out_bits,
                              void* out_logpsi, void* stream) {
  QES_ARG_CHECK(dtype == QES_DTYPE_F32 || dtype == QES_DTYPE_C64, "qes_pt_collect: bad dtype");
  QES_ARG_CHECK(n_replicas >= 1 && n_chains >= 0 && ns > 0, "qes_pt_collect: bad sizes");
  if (n_chains == 0) return QES_OK;
  QES_ARG_CHECK(chain_beta && chain_bits && logpsi && out_bits, "qes_pt_collect: null pointer");
  const int bs = 128;
  if (dtype == QES_DTYPE_F32)
    pt_collect_kernel<float><<<(n_chains + bs - 1) / bs, bs, 0, (cudaStream_t)stream>>>(
        n_replicas, n_chains, n_words(ns), chain_beta, target_beta, chain_bits, (const float*)logpsi, out_bits,
        (float*)out_logpsi);
  else
    pt_collect_kernel<float2><<<(n_chains + bs - 1) / bs, bs, 0, (cudaStream_t)stream>>>(
        n_replicas, n_chains, n_words(ns), chain_beta, target_beta, chain_bits, (const float2*)logpsi, out_bits,
        (float2*)out_logpsi);
  QES_LAUNCH_CHECK();
  return QES_OK;
}

// ----------------------------------------------------------------------------
// Batched problems: persistent warps take (problem, chain) items from a
// device queue, heaviest first, so problems of uneven size share one launch.
// ----------------------------------------------------------------------------
template <class T, int MPL>
__global__ void batch_sampler_kernel(const qes_batch_instance* __restrict__ inst, int n_items,
                                     const int4* __restrict__ items, int thermalize, float beta_mu,
                                     int recompute_every, const T* __restrict__ params,
                                     const T* __restrict__ flipC, const T* __restrict__ flipS,
                                     uint32_t* __restrict__ chain_bits, uint64_t* __restrict__ chain_step,
                                     int32_t* __restrict__ proposed, int32_t* __restrict__ accepted,
                                     uint32_t* __restrict__ sample_bits, T* __restrict__ sample_logpsi,
                                     T* __restrict__ last_logpsi, unsigned int* __restrict__ counter) {
  extern __shared__ uint32_t batch_cfg_sm[];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  uint32_t* cw = batch_cfg_sm + wid * SMP_MAX_WORDS;
  for (;;) {
    unsigned int q = 0;
    if (lane == 0) q = atomicAdd(counter, 1u);
    q = __shfl_sync(0xffffffffu, q, 0);
    if (q >= (unsigned int)n_items) break;
    const int4 it = items[q];
    const qes_batch_instance I = inst[it.x];
    ChainCtx<T> P;
    P.ns = I.ns; P.nh = I.nh; P.n_chains = I.n_chains; P.deg = 0; P.sweep_steps = I.sweep_steps;
    P.recompute_every = recompute_every; P.num_samples = I.num_samples;
    P.therm_steps_total = thermalize ? I.therm_steps_total : 0; P.beta_mu = beta_mu;
    P.k0 = (uint32_t)(I.seed & 0xffffffffu); P.k1 = (uint32_t)(I.seed >> 32);
    P.chain_id = it.y;
    P.a = params + I.param_off; P.b = P.a + I.ns; P.W = P.b + I.nh;
    P.flipC = flipC + I.flip_off; P.flipS = flipS + I.flip_off;
    P.pairC = nullptr; P.pairS = nullptr; P.nbr = nullptr; P.nbr_pair = nullptr; P.pair_i = nullptr;
    P.pair_j = nullptr;
    run_chain<T, MPL, QES_RULE_LOCAL>(P, it.y, cw, nullptr, chain_bits + I.chain_word_off, chain_step + I.chain_off,
                                      proposed + I.chain_off, accepted + I.chain_off,
                                      sample_bits + I.sample_word_off,
                                      sample_logpsi ? sample_logpsi + I.sample_off : nullptr,
                                      last_logpsi ? last_logpsi + I.chain_off : nullptr);
  }
}

template <class T, int MPL>
static int launch_batch_sampler_mpl(int n_inst, const qes_batch_instance* inst, int n_items, const int32_t* items,
                                    int warps, int blocks, int thermalize, float beta_mu, int recompute_every,
                                    const void* params, const void* flipC, const void* flipS, uint32_t* chain_bits,
                                    uint64_t* chain_step, int32_t* proposed, int32_t* accepted,
                                    uint32_t* sample_bits, void* sample_logpsi, void* last_logpsi,
                                    unsigned int* counter, cudaStream_t st) {
  (void)n_inst;
  cudaFuncAttributes fa;
  QES_CUDA_CHECK(cudaFuncGetAttributes(&fa, batch_sampler_kernel<T, MPL>));
  if (32 * warps > fa.maxThreadsPerBlock) {
    qes_set_last_message("qes_batch_sampler_run: warps_per_block exceeds the kernel's register-limited block size");
    return QES_ERR_ARG;
  }
  QES_CUDA_CHECK(cudaMemsetAsync(counter, 0, sizeof(unsigned int), st));
  const size_t smem = (size_t)warps * SMP_MAX_WORDS * sizeof(uint32_t);
  batch_sampler_kernel<T, MPL><<<blocks, 32 * warps, smem, st>>>(
      inst, n_items, (const int4*)items, thermalize, beta_mu, recompute_every, (const T*)params, (const T*)flipC,
      (const T*)flipS, chain_bits, chain_step, proposed, accepted, sample_bits, (T*)sample_logpsi, (T*)last_logpsi,
      counter);
  QES_LAUNCH_CHECK();
  return QES_OK;
}

extern "C" int qes_batch_sampler_run(int dtype, int n_inst, const qes_batch_instance* inst, int max_nh,
                                     int n_items, const int32_t* items, int warps_per_block, int n_blocks,
                                     int thermalize, float mu, float beta, int recompute_every,
                                     const void* params, const void* flipCt, const void* flipSt,
                                     uint32_t* chain_bits, uint64_t* chain_step, int32_t* proposed,
                                     int32_t* accepted, uint32_t* sample_bits, void* sample_logpsi,
                                     void* last_logpsi, unsigned int* counter, void* stream) {
  QES_ARG_CHECK(dtype == QES_DTYPE_F32 || dtype == QES_DTYPE_C64, "qes_batch_sampler_run: bad dtype");
  QES_ARG_CHECK(n_inst >= 0 && n_items >= 0 && max_nh > 0, "qes_batch_sampler_run: bad sizes");
  QES_ARG_CHECK(warps_per_block >= 1 && warps_per_block <= 16 && n_blocks >= 1,
                "qes_batch_sampler_run: warps_per_block must be 1..16 and n_blocks >= 1");
  if (n_items == 0) return QES_OK;
  QES_ARG_CHECK(inst && items && params && flipCt && flipSt && chain_bits && chain_step && proposed && accepted &&
                    sample_bits && counter,
                "qes_batch_sampler_run: null pointer");
  cudaStream_t st = (cudaStream_t)stream;
  const float bm = beta * mu;
  const int mpl = (max_nh + 31) / 32;
#define QES_BSMP_CASE(TT, M)                                                                                      \
  if (mpl <= M)                                                                                                  \
    return launch_batch_sampler_mpl<TT, M>(n_inst, inst, n_items, items, warps_per_block, n_blocks, thermalize, bm, \
                                           recompute_every, params, flipCt, flipSt, chain_bits, chain_step,      \
                                           proposed, accepted, sample_bits, sample_logpsi, last_logpsi, counter, st);
  if (dtype == QES_DTYPE_F32) {
    QES_BSMP_CASE(float, 1)
    QES_BSMP_CASE(float, 2)
    QES_BSMP_CASE(float, 4)
    QES_BSMP_CASE(float, 8)
    QES_BSMP_CASE(float, 16)
    QES_BSMP_CASE(float, 32)
    QES_BSMP_CASE(float, 64)
  } else {
    QES_BSMP_CASE(float2, 1)
    QES_BSMP_CASE(float2, 2)
    QES_BSMP_CASE(float2, 4)
    QES_BSMP_CASE(float2, 8)
    QES_BSMP_CASE(float2, 16)
  }
#undef QES_BSMP_CASE
  qes_set_last_message("qes_batch_sampler_run: too many hidden units for the register-resident theta cache");
  return QES_ERR_SIZE;
}
