// Per-voxel STZ barrier / Arrhenius rate kernels and KMC event selection.
//
// Restates mgkmc/kmc_simulator_functions.py (2D) and mgkmc/stz/{barriers,
// kmc,cascade}.py (3D).  Floating-point operation order follows the
// reference where it decides bits: contractions are left-to-right sums from
// 0.0 over (i, j) in C order, products are rounded separately (no FMA
// contraction, mirroring the LLVM code numba emits), and the total rate is
// the sequential left-to-right FP64 running sum in (x, y[, z], m) order.
//
// The sequential sum is a dependent chain by definition; it is reproduced
// bit for bit by exact integer arithmetic inside binades (see the exact
// running sum below), in parallel over chunks.  The prefix array it writes
// is monotone (rates >= 0), so selection is a two-level parallel search for
// the first prefix >= u * total instead of the reference's linear rescan;
// both return the same index for the same rates and draw.
#include <math.h>

#include <algorithm>

#include "common.cuh"

namespace mgk {

#define KB_EV 8.617e-5
#define GPA_NM3_TO_EV 6.241509

__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }

// softening base g (kmc_simulator_functions.py:114-128)
__device__ __forceinline__ double soft_base(double g_p, double g_t, double t_last, double t, double cap,
                                            double tau) {
  double g_t_curr = 0.0;
  if (g_t > 0) {
    if (isinf(tau) && tau > 0) g_t_curr = g_t;
    else if (t_last == -INFINITY) g_t_curr = 0.0;
    else {
      double dt = sub(t, t_last);
      if (dt < 0) dt = 0;
      g_t_curr = mul(g_t, exp(-__ddiv_rn(dt, tau)));
    }
  }
  double g = add(g_p, g_t_curr);
  if (cap > 0 && g > cap) g = cap;
  return g;
}

// One thread per (voxel, mode).  D = 2 or 3 (tensor dimension); SP = soft_prop
// stride (2 in 2D, 4 in 3D).
template <int D, int SP>
__device__ __forceinline__ double barrier_mode(long long i, int M, double* __restrict__ Q,
                                               const double* __restrict__ Q0, const double* __restrict__ sig,
                                               const double* __restrict__ cat, double volume,
                                               const double* __restrict__ soft, const double* __restrict__ t_last,
                                               double t, const double* __restrict__ prev, double cap, int scheme,
                                               double tau) {
  const long long v = i / M;
  const double g_base = soft_base(soft[SP * v], soft[SP * v + 1], t_last[v], t, cap, tau);
  const double* c = cat + i * D * D;
  const double* s = sig + v * D * D;
  double modifier = 1.0;
  if (scheme == 1) {
    const double* p = prev + v * D * D;
    double dot = 0.0, nm = 0.0, np = 0.0;
#pragma unroll
    for (int q = 0; q < D * D; ++q) {
      const double a = c[q], b = p[q];
      dot = add(dot, mul(a, b));
      nm = add(nm, mul(a, a));
      np = add(np, mul(b, b));
    }
    const double norm_p = sqrt(np), norm_m = sqrt(nm);
    if (norm_p < 1e-12 || norm_m < 1e-12) modifier = 1.0;
    else {
      const double ct = __ddiv_rn(dot, mul(norm_m, norm_p));
      const double o = add(1.0, ct);
      modifier = __ddiv_rn(mul(o, o), 4.0);
    }
  }
  const double g_eff = mul(modifier, g_base);
  double w = 0.0;
#pragma unroll
  for (int q = 0; q < D * D; ++q) w = add(w, mul(s[q], c[q]));
  const double w_val = mul(mul(mul(0.5, volume), __ddiv_rn(w, 1e9)), GPA_NM3_TO_EV);
  const double q = sub(mul(Q0[i], exp(-g_eff)), w_val);
  Q[i] = q;
  return q;
}

template <int D, int SP>
__global__ void barrier_kernel(long long nvox, int M, double* __restrict__ Q, const double* __restrict__ Q0,
                               const double* __restrict__ sig, const double* __restrict__ cat, double volume,
                               const double* __restrict__ soft, const double* __restrict__ t_last, double t,
                               const double* __restrict__ prev, double cap, int scheme, double tau) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= nvox * M) return;
  barrier_mode<D, SP>(i, M, Q, Q0, sig, cat, volume, soft, t_last, t, prev, cap, scheme, tau);
}

// rate of one mode (kmc_simulator_functions.py:41-48)
__device__ __forceinline__ double mode_rate(double q, double beta, double vnu) {
  return q <= 0 ? vnu : mul(vnu, exp(-mul(q, beta)));
}

__device__ __forceinline__ double beta_of(double T) { return T > 0.0 ? __ddiv_rn(1.0, mul(KB_EV, T)) : INFINITY; }

// Fused barrier, rate and block-sum pass (fast selection mode): the barriers
// as barrier_kernel, each mode's KMC-mode rate from its new barrier, and the
// FP64 sum of the rates per CTA (grid-stride, fixed grid: a deterministic
// order); no rate array is written.
template <int D, int SP>
__global__ void __launch_bounds__(256) barrier_total_kernel(long long nvox, int M, double* __restrict__ Q,
                                                            const double* __restrict__ Q0,
                                                            const double* __restrict__ sig,
                                                            const double* __restrict__ cat, double volume,
                                                            const double* __restrict__ soft,
                                                            const double* __restrict__ t_last, double t,
                                                            const double* __restrict__ prev, double cap, int scheme,
                                                            double tau, const double* __restrict__ T, double Ts,
                                                            double vnu, double* __restrict__ partials) {
  __shared__ double red[32];
  const double beta_s = beta_of(Ts);
  double acc = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nvox * M;
       i += (long long)gridDim.x * blockDim.x) {
    const double q = barrier_mode<D, SP>(i, M, Q, Q0, sig, cat, volume, soft, t_last, t, prev, cap, scheme, tau);
    acc += mode_rate(q, T ? beta_of(T[i / M]) : beta_s, vnu);
  }
  acc = block_sum(acc, red);
  if (threadIdx.x == 0) partials[blockIdx.x] = acc;
}

// sum of nb partials in a fixed order (one CTA)
__global__ void __launch_bounds__(256) partials_total_kernel(const double* __restrict__ partials, int nb,
                                                             double* __restrict__ d_total) {
  __shared__ double red[32];
  double acc = 0.0;
  for (int k = threadIdx.x; k < nb; k += blockDim.x) acc += partials[k];
  acc = block_sum(acc, red);
  if (threadIdx.x == 0) *d_total = acc;
}

// Non-compacting rates (KMC mode: every mode is an event).
__global__ void rates_full_kernel(long long nvox, int M, const double* __restrict__ Q, double vnu,
                                  const double* __restrict__ T, double Ts, double* __restrict__ rates,
                                  long long* __restrict__ indices, long long* __restrict__ d_count) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i == 0 && d_count) *d_count = nvox * M;
  if (i >= nvox * M) return;
  const long long v = i / M;
  const double beta = beta_of(T ? T[v] : Ts);
  rates[i] = mode_rate(Q[i], beta, vnu);
  if (indices) indices[i] = i;
}

// Compacting rates (cascade mode: only q > 0), 3 passes: block counts,
// exclusive scan of the counts, ordered scatter.
__global__ void rates_count_kernel(long long n, const double* __restrict__ Q, int* __restrict__ bcount) {
  __shared__ int red[32];
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  int f = (i < n && Q[i] > 0) ? 1 : 0;
  int s = block_sum(f, red);
  if (threadIdx.x == 0) bcount[blockIdx.x] = s;
}

__global__ void scan_counts_kernel(int nb, int* __restrict__ bcount, long long* __restrict__ d_count) {
  // single CTA exclusive scan over nb block counts (in place)
  __shared__ long long carry;
  __shared__ int wsum[32];
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int base = 0; base < nb; base += blockDim.x) {
    const int i = base + threadIdx.x;
    int v = i < nb ? bcount[i] : 0;
    // inclusive warp scan
    int x = v;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int o = 1; o < 32; o <<= 1) { int y = __shfl_up_sync(0xffffffffu, x, o); if (lane >= o) x += y; }
    if (lane == 31) wsum[wid] = x;
    __syncthreads();
    if (wid == 0) {
      int w = lane < (int)(blockDim.x >> 5) ? wsum[lane] : 0;
      for (int o = 1; o < 32; o <<= 1) { int y = __shfl_up_sync(0xffffffffu, w, o); if (lane >= o) w += y; }
      wsum[lane] = w;
    }
    __syncthreads();
    const int incl = x + (wid > 0 ? wsum[wid - 1] : 0);
    if (i < nb) bcount[i] = (int)(carry + incl - v);
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) carry += incl;
    __syncthreads();
  }
  if (threadIdx.x == 0) *d_count = carry;
}

__global__ void rates_scatter_kernel(long long nvox, int M, const double* __restrict__ Q, double vnu,
                                     const double* __restrict__ T, double Ts, const int* __restrict__ boff,
                                     double* __restrict__ rates, long long* __restrict__ indices) {
  __shared__ int wsum[32];
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long n = nvox * M;
  const double q = i < n ? Q[i] : 0.0;
  const int f = (i < n && q > 0) ? 1 : 0;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int x = f;
  for (int o = 1; o < 32; o <<= 1) { int y = __shfl_up_sync(0xffffffffu, x, o); if (lane >= o) x += y; }
  if (lane == 31) wsum[wid] = x;
  __syncthreads();
  if (wid == 0) {
    int w = lane < (int)(blockDim.x >> 5) ? wsum[lane] : 0;
    for (int o = 1; o < 32; o <<= 1) { int y = __shfl_up_sync(0xffffffffu, w, o); if (lane >= o) w += y; }
    wsum[lane] = w;
  }
  __syncthreads();
  if (!f) return;
  const long long pos = (long long)boff[blockIdx.x] + x - 1 + (wid > 0 ? wsum[wid - 1] : 0);
  const double beta = beta_of(T ? T[i / M] : Ts);
  rates[pos] = mode_rate(q, beta, vnu);
  indices[pos] = i;
}

// Exact sequential running sum, computed in parallel.
//
// The reference accumulates total_rate left to right in FP64
// (kmc_simulator_functions.py:36-55), so every running sum carries the
// rounding of all earlier additions.  Rates are >= 0, so the running sum s
// only grows.  While s stays inside one binade [2^e, 2^(e+1)), every double
// there is a multiple of u = 2^(e-52), and round-to-nearest of s + r is
// s + rint(r/u)*u unless r/u sits exactly halfway between integers (a tie,
// whose rounding depends on the parity of s).  So over a run of rates the
// chain collapses to an exact int64 prefix sum of q_i = rint(r_i/u) added to
// the mantissa integer M = s/u, valid up to the first element whose candidate
// leaves the binade (M + Q >= 2^53) or is a tie; that element is added the
// ordinary way (one __dadd_rn), which moves s to its new binade.  A zero,
// subnormal or non-finite s also takes single ordinary adds.  The results
// are bit-identical to the sequential loop.
//
// The array is cut into chunks of kExactChunk rates, processed in five
// launches:
//   1. chunk sums in FP64, any order (an estimate of the running sum);
//   2. one CTA scans them: the estimated running sum at each chunk start;
//   3. per chunk, with the binade e of that estimate: the exact int64 sum Q
//      of q_i, and whether every element is representable and tie-free;
//   4. one CTA walks the chunks in order with the exact running sum s: a
//      chunk whose record holds (s in binade e, M + Q < 2^53) ends at
//      (M + Q) u exactly and costs a few instructions; any other chunk (the
//      first, the last short one, a binade crossing, a tie, a wrong estimate)
//      runs the sequential-exact CTA algorithm above on its own rates;
//   5. per chunk that the walk accepted: prefix_i = (M + Q_i) u from a block
//      scan of its q_i.
// A chunk's records sit in its own first four prefix entries until the walk
// (rejected chunks) or launch 5 (accepted ones) writes its final values; the
// walk marks accepted chunks with -0.0 in entry 3, a value no running sum
// from +0.0 can take.  The walk's cost is about the number of binades the
// sum crosses, times one chunk.
constexpr int kExactThreads = 1024;
constexpr int kExactPer = 8;  // rates per thread per chunk
constexpr int kExactChunk = kExactThreads * kExactPer;
// q_i < 2^53, so sums of q are saturated at 2^61 (no int64 overflow); any
// saturated sum is far above 2^53 - M and reads as leaving the binade
constexpr long long kQCap = 1LL << 61;
__device__ __forceinline__ long long qsat(long long a, long long b) { return min(a + b, kQCap); }
constexpr long long kRecOk = 1LL << 62;                      // record tag: chunk tie-free, q representable
constexpr long long kRecMark = (long long)0x8000000000000000ULL;  // bits of -0.0: accepted by the walk

__device__ __forceinline__ bool normal_finite(double s) { return s >= 2.2250738585072014e-308 && s < 1.0 / 0.0; }
__device__ __forceinline__ int binade_of(double s) { return (int)((__double_as_longlong(s) >> 52) & 0x7ff) - 1023; }

// The sequential-exact algorithm on rates[p0, end) from running sum s0, by
// all kExactThreads threads of the CTA; writes prefix[p0, end) and returns
// the running sum after element end - 1 (in every thread).
__device__ double exact_range(const double* __restrict__ rates, long long p0, long long end, double s0,
                              double* __restrict__ prefix, long long* w_sum, long long* w_fail, double* s_s,
                              long long* s_p) {
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  __syncthreads();
  if (tid == 0) { *s_s = s0; *s_p = p0; }
  __syncthreads();
  while (true) {
    const double s = *s_s;
    const long long p = *s_p;
    if (p >= end) break;
    if (!normal_finite(s)) {
      // zero, subnormal or non-finite running sum: one ordinary add
      __syncthreads();
      if (tid == 0) {
        const double v = add(s, rates[p]);
        prefix[p] = v;
        *s_s = v;
        *s_p = p + 1;
      }
      __syncthreads();
      continue;
    }
    const long long bits = __double_as_longlong(s);
    const int e = binade_of(s);
    const long long M = (bits & ((1LL << 52) - 1)) | (1LL << 52);
    const double scale = ldexp(1.0, 52 - e);  // 1/u, exact power of two
    const double u = ldexp(1.0, e - 52);
    const long long base = p + (long long)tid * kExactPer;
    long long q[kExactPer];
    long long fail = LLONG_MAX;  // first tie or unrepresentable element of this thread
    long long tot = 0;
#pragma unroll
    for (int k = 0; k < kExactPer; ++k) {
      const long long i = base + k;
      q[k] = 0;
      if (i < end) {
        const double x = rates[i] * scale;
        if (!(x >= 0.0) || !(x < 9007199254740992.0) || x - floor(x) == 0.5) {
          if (fail == LLONG_MAX) fail = i;
        } else {
          q[k] = (long long)rint(x);
        }
      }
      tot += q[k];
    }
    // exclusive block scan of the per-thread totals (int64, exact)
    long long incl = tot;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const long long t = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl = qsat(incl, t);
    }
    long long wf = fail;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) wf = min(wf, __shfl_xor_sync(0xffffffffu, wf, o));
    if (lane == 31) w_sum[wid] = incl;
    if (lane == 0) w_fail[wid] = wf;
    __syncthreads();
    if (wid == 0) {
      long long v = w_sum[lane];
      long long f = w_fail[lane];
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const long long t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v = qsat(v, t);
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) f = min(f, __shfl_xor_sync(0xffffffffu, f, o));
      w_sum[lane] = v;  // inclusive warp totals
      if (lane == 0) w_fail[0] = f;
    }
    __syncthreads();
    // before this thread's first element (a saturated incl minus tot stays far above 2^53)
    long long Q = qsat(wid > 0 ? w_sum[wid - 1] : 0, incl - tot);
    long long first_bad = w_fail[0];
    // first element whose candidate leaves the binade (Q is nondecreasing)
    long long cross = LLONG_MAX;
#pragma unroll
    for (int k = 0; k < kExactPer; ++k) {
      const long long i = base + k;
      if (i < end && i < first_bad) {
        Q = qsat(Q, q[k]);
        if (M + Q >= (1LL << 53)) { cross = i; break; }
        prefix[i] = (double)(M + Q) * u;
      }
    }
    // the step is valid up to min(first tie, first crossing)
    long long wc = cross;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) wc = min(wc, __shfl_xor_sync(0xffffffffu, wc, o));
    __syncthreads();  // everyone has read w_fail[0]
    if (lane == 0) w_sum[wid] = wc;
    __syncthreads();
    if (tid == 0) {
      long long stop = first_bad;
      for (int w = 0; w < kExactThreads / 32; ++w) stop = min(stop, w_sum[w]);
      const long long stp_end = min(p + (long long)kExactChunk, end);
      if (stop >= stp_end) {
        // whole step valid: the running sum is its last prefix
        *s_s = prefix[stp_end - 1];
        *s_p = stp_end;
      } else {
        // elements [p, stop) were written; stop is added the ordinary way
        const double prev = stop > p ? prefix[stop - 1] : s;
        const double v = add(prev, rates[stop]);
        prefix[stop] = v;
        *s_s = v;
        *s_p = stop + 1;
      }
    }
    __syncthreads();
  }
  return *s_s;
}

__device__ __forceinline__ long long exact_count(long long n_fixed, const long long* d_count) {
  return d_count ? *d_count : n_fixed;
}
// chunks that carry records: not the first, at least 4 rates long
__device__ __forceinline__ bool has_record(long long c0, long long n) { return c0 > 0 && n - c0 >= 4; }

__device__ __forceinline__ double block_sum_d(double v, double* red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double t = 0;
  if (threadIdx.x < 32) {
    t = threadIdx.x < (blockDim.x + 31) / 32 ? red[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
  }
  return t;  // valid in thread 0
}

// 1. FP64 sum of each chunk (an estimate) into the chunk's entry 0; grid = chunks
__global__ void __launch_bounds__(256) exact_chunk_sum_kernel(const double* __restrict__ rates, long long n_fixed,
                                                              const long long* __restrict__ d_count,
                                                              double* __restrict__ prefix) {
  __shared__ double red[32];
  const long long n = exact_count(n_fixed, d_count);
  const long long c0 = (long long)blockIdx.x * kExactChunk;
  if (c0 >= n || n - c0 < 4) return;  // the last short chunk needs no estimate
  const long long c1 = min(c0 + (long long)kExactChunk, n);
  double v = 0;
  for (long long i = c0 + threadIdx.x; i < c1; i += blockDim.x) v += rates[i];
  v = block_sum_d(v, red);
  if (threadIdx.x == 0) prefix[c0] = v;
}

// 2. one CTA: estimated running sum at each chunk start into entry 1
__global__ void __launch_bounds__(1024) exact_chunk_scan_kernel(long long n_fixed, const long long* __restrict__ d_count,
                                                                double* __restrict__ prefix) {
  __shared__ double wtot[32];
  __shared__ double carry;
  const long long n = exact_count(n_fixed, d_count);
  const long long K = (n + kExactChunk - 1) / kExactChunk;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (threadIdx.x == 0) carry = 0.0;
  __syncthreads();
  for (long long kb = 0; kb < K; kb += 1024) {
    const long long k = kb + threadIdx.x;
    const long long c0 = k * kExactChunk;
    const double v = (k < K && n - c0 >= 4) ? prefix[c0] : 0.0;
    double incl = v;
    for (int o = 1; o < 32; o <<= 1) {
      const double t = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += t;
    }
    if (lane == 31) wtot[wid] = incl;
    __syncthreads();
    if (wid == 0) {
      double w = wtot[lane];
      for (int o = 1; o < 32; o <<= 1) {
        const double t = __shfl_up_sync(0xffffffffu, w, o);
        if (lane >= o) w += t;
      }
      wtot[lane] = w;
    }
    __syncthreads();
    const double excl = carry + (wid > 0 ? wtot[wid - 1] : 0.0) + (incl - v);
    if (k < K && has_record(c0, n)) prefix[c0 + 1] = excl;
    __syncthreads();
    if (threadIdx.x == 0) carry += wtot[31];
    __syncthreads();
  }
}

// q_i = rint(r_i * scale) of rate i, or -1 when it is a tie or not
// representable (then the chunk is left to the sequential algorithm)
__device__ __forceinline__ long long exact_q(double r, double scale) {
  const double x = r * scale;
  if (!(x >= 0.0) || !(x < 9007199254740992.0) || x - floor(x) == 0.5) return -1;
  return (long long)rint(x);
}

// 3. per chunk with a record: Q = sum of q_i at the binade of its estimated
// start (entry 2), and the tag with that binade (entry 3); grid = chunks
__global__ void __launch_bounds__(kExactThreads) exact_chunk_q_kernel(const double* __restrict__ rates,
                                                                      long long n_fixed,
                                                                      const long long* __restrict__ d_count,
                                                                      double* __restrict__ prefix) {
  __shared__ long long w_q[32];
  __shared__ int w_bad[32];
  __shared__ double s_est;
  const long long n = exact_count(n_fixed, d_count);
  const long long c0 = (long long)blockIdx.x * kExactChunk;
  if (c0 >= n || !has_record(c0, n)) return;
  const long long c1 = min(c0 + (long long)kExactChunk, n);
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  if (tid == 0) s_est = prefix[c0 + 1];
  __syncthreads();
  const double est = s_est;
  const bool est_ok = normal_finite(est);
  const int e = est_ok ? binade_of(est) : 0;
  const double scale = ldexp(1.0, 52 - e);
  long long tot = 0;
  int bad = est_ok ? 0 : 1;
  const long long base = c0 + (long long)tid * kExactPer;
#pragma unroll
  for (int k = 0; k < kExactPer; ++k) {
    const long long i = base + k;
    if (i < c1 && !bad) {
      const long long q = exact_q(rates[i], scale);
      if (q < 0) bad = 1;
      else tot = qsat(tot, q);
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    tot = qsat(tot, __shfl_xor_sync(0xffffffffu, tot, o));
    bad |= __shfl_xor_sync(0xffffffffu, bad, o);
  }
  if (lane == 0) { w_q[wid] = tot; w_bad[wid] = bad; }
  __syncthreads();  // every thread has read entry 1 (s_est) before entry 2/3 change
  if (tid == 0) {
    long long Q = 0;
    int b = 0;
    for (int w = 0; w < kExactThreads / 32; ++w) { Q = qsat(Q, w_q[w]); b |= w_bad[w]; }
    prefix[c0 + 2] = __longlong_as_double(Q);
    prefix[c0 + 3] = __longlong_as_double(b ? 0LL : (kRecOk | (long long)(e + 2048)));
  }
}

// 4. one CTA walks the chunks in order with the exact running sum; writes the
// total.  Accepted chunks get (M, e, mark) in entries 0, 1, 3.
__global__ void __launch_bounds__(kExactThreads) exact_walk_kernel(const double* __restrict__ rates, long long n_fixed,
                                                                   const long long* __restrict__ d_count,
                                                                   double* __restrict__ prefix,
                                                                   double* __restrict__ d_total) {
  __shared__ long long w_sum[32];
  __shared__ long long w_fail[32];
  __shared__ double s_s;
  __shared__ long long s_p;
  __shared__ long long rec_q[kExactThreads];
  __shared__ long long rec_t[kExactThreads];
  __shared__ double w_s;
  __shared__ long long w_k;
  const long long n = exact_count(n_fixed, d_count);
  const long long K = (n + kExactChunk - 1) / kExactChunk;
  double s = 0.0;
  for (long long kb = 0; kb < K; kb += kExactThreads) {
    const long long kend = min(kb + (long long)kExactThreads, K);
    {
      const long long k = kb + threadIdx.x;
      const long long c0 = k * kExactChunk;
      const bool rec = k < kend && has_record(c0, n);
      rec_q[threadIdx.x] = rec ? __double_as_longlong(prefix[c0 + 2]) : 0;
      rec_t[threadIdx.x] = rec ? __double_as_longlong(prefix[c0 + 3]) : 0;
    }
    __syncthreads();
    long long k = kb;
    while (k < kend) {
      if (threadIdx.x == 0) {
        // accept chunks while their records hold at the exact running sum
        while (k < kend) {
          const long long c0 = k * kExactChunk;
          const long long t = rec_t[k - kb];
          if (!has_record(c0, n) || !(t & kRecOk) || !normal_finite(s)) break;
          const int e = (int)(t & 0xffff) - 2048;
          if (binade_of(s) != e) break;
          const long long M = (__double_as_longlong(s) & ((1LL << 52) - 1)) | (1LL << 52);
          const long long Q = rec_q[k - kb];
          if (M + Q >= (1LL << 53)) break;
          prefix[c0] = __longlong_as_double(M);
          prefix[c0 + 1] = __longlong_as_double((long long)e);
          prefix[c0 + 3] = __longlong_as_double(kRecMark);
          s = (double)(M + Q) * ldexp(1.0, e - 52);
          ++k;
        }
        w_s = s;
        w_k = k;
      }
      __syncthreads();
      s = w_s;
      k = w_k;
      if (k < kend) {
        // chunk k by the sequential-exact algorithm
        const long long c0 = k * kExactChunk;
        s = exact_range(rates, c0, min(c0 + (long long)kExactChunk, n), s, prefix, w_sum, w_fail, &s_s, &s_p);
        ++k;
      }
      __syncthreads();
    }
  }
  if (threadIdx.x == 0) *d_total = n > 0 ? s : 0.0;
}

// 5. per accepted chunk: prefix_i = (M + Q_i) u, Q_i the inclusive sum of q
// up to i; grid = chunks
__global__ void __launch_bounds__(kExactThreads) exact_write_kernel(const double* __restrict__ rates, long long n_fixed,
                                                                    const long long* __restrict__ d_count,
                                                                    double* __restrict__ prefix) {
  __shared__ long long w_sum[32];
  __shared__ long long s_rec[3];
  const long long n = exact_count(n_fixed, d_count);
  const long long c0 = (long long)blockIdx.x * kExactChunk;
  if (c0 >= n || !has_record(c0, n)) return;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  if (tid < 3) s_rec[tid] = __double_as_longlong(prefix[c0 + (tid == 2 ? 3 : tid)]);
  __syncthreads();
  if (s_rec[2] != kRecMark) return;  // the walk wrote this chunk
  const long long M = s_rec[0];
  const int e = (int)s_rec[1];
  const long long c1 = min(c0 + (long long)kExactChunk, n);
  const double scale = ldexp(1.0, 52 - e), u = ldexp(1.0, e - 52);
  const long long base = c0 + (long long)tid * kExactPer;
  long long q[kExactPer];
  long long tot = 0;
#pragma unroll
  for (int k = 0; k < kExactPer; ++k) {
    const long long i = base + k;
    q[k] = i < c1 ? exact_q(rates[i], scale) : 0;  // >= 0: the chunk's record said so
    tot += q[k];
  }
  long long incl = tot;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const long long t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  if (lane == 31) w_sum[wid] = incl;
  __syncthreads();
  if (wid == 0) {
    long long v = w_sum[lane];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const long long t = __shfl_up_sync(0xffffffffu, v, o);
      if (lane >= o) v += t;
    }
    w_sum[lane] = v;
  }
  __syncthreads();
  long long Q = (wid > 0 ? w_sum[wid - 1] : 0) + (incl - tot);
#pragma unroll
  for (int k = 0; k < kExactPer; ++k) {
    const long long i = base + k;
    if (i < c1) {
      Q += q[k];
      prefix[i] = (double)(M + Q) * u;
    }
  }
}

// the five launches for up to n_max rates (the count is *d_count when given)
static int launch_exact_prefix(const double* rates, long long n_max, const long long* d_count, double* prefix,
                               double* d_total, cudaStream_t s) {
  const long long nfix = d_count ? 0 : n_max;
  const unsigned int K = (unsigned int)std::max(1LL, (n_max + kExactChunk - 1) / kExactChunk);
  exact_chunk_sum_kernel<<<K, 256, 0, s>>>(rates, nfix, d_count, prefix);
  exact_chunk_scan_kernel<<<1, 1024, 0, s>>>(nfix, d_count, prefix);
  exact_chunk_q_kernel<<<K, kExactThreads, 0, s>>>(rates, nfix, d_count, prefix);
  exact_walk_kernel<<<1, kExactThreads, 0, s>>>(rates, nfix, d_count, prefix, d_total);
  exact_write_kernel<<<K, kExactThreads, 0, s>>>(rates, nfix, d_count, prefix);
  MGK_CUDA(cudaGetLastError());
  return MGK_OK;
}

// First i with prefix[i] >= u*total (two-level parallel search, one CTA).
__global__ void select_kernel(const double* __restrict__ prefix, const long long* __restrict__ d_count,
                              const double* __restrict__ d_total, double u, long long* __restrict__ d_index) {
  __shared__ long long best;
  const long long n = *d_count;
  const double total = *d_total;
  if (threadIdx.x == 0) best = LLONG_MAX;
  __syncthreads();
  if (!(total > 0) || n <= 0) {
    // total <= 0 -> -1 (kmc_simulator_functions.py:61); NaN total scans to the end
    if (threadIdx.x == 0) *d_index = (total <= 0 || n <= 0) ? -1 : n - 1;
    return;
  }
  const double r = add(0.0, mul(sub(total, 0.0), u));
  const long long T = blockDim.x;
  const long long stride = (n + T - 1) / T;
  // level 1: sample the last element of each stride segment
  const long long seg_end = min(n, (threadIdx.x + 1) * stride) - 1;
  if (threadIdx.x * stride < n && prefix[seg_end] >= r) atomicMin((unsigned long long*)&best, (unsigned long long)threadIdx.x);
  __syncthreads();
  const long long seg = best;
  __syncthreads();
  if (threadIdx.x == 0) best = LLONG_MAX;
  __syncthreads();
  if (seg == LLONG_MAX) {
    if (threadIdx.x == 0) *d_index = n - 1;
    return;
  }
  const long long lo = seg * stride, hi = min(n, lo + stride);
  for (long long i = lo + threadIdx.x; i < hi; i += T)
    if (prefix[i] >= r) atomicMin((unsigned long long*)&best, (unsigned long long)i);
  __syncthreads();
  if (threadIdx.x == 0) *d_index = best == LLONG_MAX ? n - 1 : best;
}

// apply_flip_soa_2d (kmc_simulator_functions.py:183-218), one thread.
__global__ void flip2d_kernel(int nx, int ny, int M, double* ep, double* soft, double* tl, const double* cat, int x,
                              int y, int m, double t, double jp, double jt, double gmax, double jn) {
  const long long v = (long long)x * ny + y;
  const double* c = cat + ((v * M) + m) * 4;
  for (int q = 0; q < 4; ++q) ep[4 * v + q] = add(ep[4 * v + q], c[q]);
  const double e11 = c[0], e22 = c[3], e12 = c[1];
  const double d = sub(e11, e22);
  const double s = add(mul(e12, e12), __ddiv_rn(add(add(mul(e22, e22), mul(e11, e11)), mul(d, d)), 6.0));
  double gp = add(soft[2 * v], mul(jp, s));
  if (gmax > 0 && gp > gmax) gp = gmax;
  soft[2 * v] = gp;
  soft[2 * v + 1] = mul(jt, s);
  tl[v] = t;
  if (jn > 0.0) {
    for (int dx = -1; dx <= 1; ++dx)
      for (int dy = -1; dy <= 1; ++dy) {
        if (dx == 0 && dy == 0) continue;
        const long long w = (long long)((x + dx + nx) % nx) * ny + (y + dy + ny) % ny;
        double g = add(soft[2 * w], mul(mul(jn, jp), s));
        if (gmax > 0 && g > gmax) g = gmax;
        soft[2 * w] = g;
        soft[2 * w + 1] = add(soft[2 * w + 1], mul(mul(jn, jt), s));
      }
  }
}

// apply_flip_soa (mgkmc/stz/cascade.py:43-111), one thread.
// apply_flip_soa (stz/cascade.py:43-111) at voxel v = (x, y, z), mode m:
// eps_p += C, softening from sum_sq, 26-neighbour fraction when jn > 0.
__device__ void flip3d_body(int nx, int ny, int nz, int M, double* ep, double* soft, double* tl, const double* cat,
                            int x, int y, int z, int m, double t, double jp, double jt, double gmax, double jn) {
  const long long v = ((long long)x * ny + y) * nz + z;
  const double* c = cat + ((v * M) + m) * 9;
  for (int q = 0; q < 9; ++q) ep[9 * v + q] = add(ep[9 * v + q], c[q]);
  const double e11 = c[0], e22 = c[4], e33 = c[8], e12 = c[1], e13 = c[2], e23 = c[5];
  const double a = sub(e22, e33), b = sub(e33, e11), d = sub(e11, e22);
  const double s = add(add(add(mul(e12, e12), mul(e23, e23)), mul(e13, e13)),
                       __ddiv_rn(add(add(mul(a, a), mul(b, b)), mul(d, d)), 6.0));
  double gp = add(soft[4 * v], mul(jp, s));
  if (gmax > 0 && gp > gmax) gp = gmax;
  soft[4 * v] = gp;
  soft[4 * v + 1] = mul(jt, s);
  tl[v] = t;
  if (jn > 0.0) {
    for (int dx = -1; dx <= 1; ++dx)
      for (int dy = -1; dy <= 1; ++dy)
        for (int dz = -1; dz <= 1; ++dz) {
          if (dx == 0 && dy == 0 && dz == 0) continue;
          const long long w = ((long long)((x + dx + nx) % nx) * ny + (y + dy + ny) % ny) * nz + (z + dz + nz) % nz;
          double g = add(soft[4 * w], mul(mul(jn, jp), s));
          if (gmax > 0 && g > gmax) g = gmax;
          soft[4 * w] = g;
          soft[4 * w + 1] = add(soft[4 * w + 1], mul(mul(jn, jt), s));
        }
  }
}

__global__ void flip3d_kernel(int nx, int ny, int nz, int M, double* ep, double* soft, double* tl, const double* cat,
                              int x, int y, int z, int m, double t, double jp, double jt, double gmax, double jn) {
  flip3d_body(nx, ny, nz, M, ep, soft, tl, cat, x, y, z, m, t, jp, jt, gmax, jn);
}

// One 3D KMC event on the device (aqs.py:889-892 selection and decode,
// :996-997 apply_flip_soa and prev_strain_dir, :1006-1013 the redraw of the
// voxel's catalog and barriers from values the host drew).  d_sel holds the
// position in the rates array; `indices` maps it to the mode index (NULL:
// identity, KMC mode).  Writes (x, y, z, m) to d_xyzm (may be NULL); a
// negative selection changes nothing and writes -1s.
__global__ void event3d_kernel(int nx, int ny, int nz, int M, const long long* d_sel, const long long* indices,
                               double* ep, double* soft, double* tl, double* cat, double* Q0, double* prev,
                               const double* new_cat, const double* new_q0, double t, double jp, double jt,
                               double gmax, double jn, long long* d_xyzm) {
  const long long k = *d_sel;
  if (k < 0) {
    if (d_xyzm) { d_xyzm[0] = -1; d_xyzm[1] = -1; d_xyzm[2] = -1; d_xyzm[3] = -1; }
    return;
  }
  const long long idx = indices ? indices[k] : k;
  const int m = (int)(idx % M);
  long long tmp = idx / M;
  const int z = (int)(tmp % nz);
  tmp /= nz;
  const int y = (int)(tmp % ny);
  const int x = (int)(tmp / ny);
  const long long v = ((long long)x * ny + y) * nz + z;
  double C[9];
  for (int q = 0; q < 9; ++q) C[q] = cat[(v * M + m) * 9 + q];
  flip3d_body(nx, ny, nz, M, ep, soft, tl, cat, x, y, z, m, t, jp, jt, gmax, jn);
  for (int q = 0; q < 9; ++q) prev[9 * v + q] = C[q];
  if (new_cat)
    for (int q = 0; q < 9 * M; ++q) cat[v * M * 9 + q] = new_cat[q];
  if (new_q0)
    for (int q = 0; q < M; ++q) Q0[v * M + q] = new_q0[q];
  if (d_xyzm) { d_xyzm[0] = x; d_xyzm[1] = y; d_xyzm[2] = z; d_xyzm[3] = m; }
}

// One KMC event on the device (kmc_simulator.py:899-900, :1025-1042): decode
// the selected mode, apply the flip bookkeeping of apply_flip_soa_2d, record
// the mode as prev_strain_dir of the voxel, and redraw the voxel's catalog and
// barriers from values the host drew.  d_sel holds the position in the rates
// array; `indices` maps it to the mode index (NULL: identity, KMC mode).
__global__ void event2d_kernel(int nx, int ny, int M, const long long* d_sel, const long long* indices,
                               double* ep, double* soft, double* tl, double* cat, double* Q0, double* prev,
                               const double* new_cat, const double* new_q0, double t, double jp, double jt,
                               double gmax, double jn, long long* d_xym) {
  const long long k = *d_sel;
  if (k < 0) {
    if (d_xym) { d_xym[0] = -1; d_xym[1] = -1; d_xym[2] = -1; }
    return;
  }
  const long long idx = indices ? indices[k] : k;
  const int m = (int)(idx % M);
  const long long tmp = idx / M;
  const int y = (int)(tmp % ny);
  const int x = (int)(tmp / ny);
  const long long v = tmp;
  double C[4];
  for (int q = 0; q < 4; ++q) C[q] = cat[(v * M + m) * 4 + q];
  for (int q = 0; q < 4; ++q) ep[4 * v + q] = add(ep[4 * v + q], C[q]);
  const double e11 = C[0], e22 = C[3], e12 = C[1];
  const double d = sub(e11, e22);
  const double s = add(mul(e12, e12), __ddiv_rn(add(add(mul(e22, e22), mul(e11, e11)), mul(d, d)), 6.0));
  double gp = add(soft[2 * v], mul(jp, s));
  if (gmax > 0 && gp > gmax) gp = gmax;
  soft[2 * v] = gp;
  soft[2 * v + 1] = mul(jt, s);
  tl[v] = t;
  if (jn > 0.0) {
    for (int dx = -1; dx <= 1; ++dx)
      for (int dy = -1; dy <= 1; ++dy) {
        if (dx == 0 && dy == 0) continue;
        const long long w = (long long)((x + dx + nx) % nx) * ny + (y + dy + ny) % ny;
        double g = add(soft[2 * w], mul(mul(jn, jp), s));
        if (gmax > 0 && g > gmax) g = gmax;
        soft[2 * w] = g;
        soft[2 * w + 1] = add(soft[2 * w + 1], mul(mul(jn, jt), s));
      }
  }
  for (int q = 0; q < 4; ++q) prev[4 * v + q] = C[q];
  if (new_cat)
    for (int q = 0; q < 4 * M; ++q) cat[v * M * 4 + q] = new_cat[q];
  if (new_q0)
    for (int q = 0; q < M; ++q) Q0[v * M + q] = new_q0[q];
  if (d_xym) { d_xym[0] = x; d_xym[1] = y; d_xym[2] = m; }
}

// Fast-patching stress update (mgkmc/kmc_simulator.py:1052-1069; cascade
// branch :764-774), one thread per voxel.  The flipped mode comes from the
// device selection (through the compacted index list when one is given), so
// the host never waits for it; a negative selection changes nothing, and a
// null selection applies only the macro-strain term.  Per component, in the
// reference's order: s + unit*scale, then every window entry gxx*K0 + gxy*K1
// that lands on this voxel in (dx, dy) order (periodic wrap: a window wider
// than the grid adds more than once), then + (gxx*m0 + gxy*m1).  Each product
// and sum is rounded on its own, as numpy evaluates the expressions.
__global__ void patch2d_kernel(int nx, int ny, int M, double* __restrict__ sig, const double* __restrict__ unit,
                               double scale, const double* __restrict__ kern, const double* __restrict__ miss,
                               int R, const double* __restrict__ cat, const long long* __restrict__ d_sel,
                               const long long* __restrict__ indices) {
  const long long nv = (long long)nx * ny;
  const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= nv) return;
  long long idx = -1;
  if (d_sel) {
    const long long k = *d_sel;
    if (k < 0) return;
    idx = indices ? indices[k] : k;
    if (idx < 0 || idx >= nv * M) return;
  }
  double2* s2 = reinterpret_cast<double2*>(sig + 4 * v);
  const double2 a = s2[0], b = s2[1];
  double s[4] = {a.x, a.y, b.x, b.y};
  if (unit) {
    const double2* u2 = reinterpret_cast<const double2*>(unit + 4 * v);
    const double2 ua = u2[0], ub = u2[1];
    s[0] = add(s[0], mul(ua.x, scale));
    s[1] = add(s[1], mul(ua.y, scale));
    s[2] = add(s[2], mul(ub.x, scale));
    s[3] = add(s[3], mul(ub.y, scale));
  }
  if (idx >= 0) {
    const long long fv = idx / M;
    const int x = (int)(fv / ny), y = (int)(fv % ny);
    const double gxx = cat[idx * 4 + 0], gxy = cat[idx * 4 + 1];
    const int i = (int)(v / ny), j = (int)(v % ny);
    const int W = 2 * R + 1;
    const int di = ((i - x) % nx + nx) % nx, dj = ((j - y) % ny + ny) % ny;
    for (int dx = di - nx * ((di + R) / nx); dx <= R; dx += nx)
      for (int dy = dj - ny * ((dj + R) / ny); dy <= R; dy += ny) {
        const double* k0 = kern + ((long long)(dx + R) * W + (dy + R)) * 4;
        const double* k1 = k0 + (long long)W * W * 4;
        for (int c = 0; c < 4; ++c) s[c] = add(s[c], add(mul(gxx, k0[c]), mul(gxy, k1[c])));
      }
    for (int c = 0; c < 4; ++c) s[c] = add(s[c], add(mul(gxx, miss[c]), mul(gxy, miss[4 + c])));
  }
  s2[0] = make_double2(s[0], s[1]);
  s2[1] = make_double2(s[2], s[3]);
}

// Stress patches from the two basis responses (kmc_simulator.py:229-261).
// Block b crops response b to the (2R+1)^2 window centred on (nx/2, ny/2) and
// writes mean(r_b) - sum(window_b) / (nx*ny) per component.  Runs once per
// simulation; 256 threads.
__global__ void patch2d_setup_kernel(int nx, int ny, int R, const double* __restrict__ r0,
                                     const double* __restrict__ r1, double* __restrict__ kern,
                                     double* __restrict__ miss) {
  __shared__ double red[4][256];
  const int b = blockIdx.x, t = threadIdx.x;
  const double* r = b ? r1 : r0;
  const long long W = 2 * R + 1, nv = (long long)nx * ny;
  double* kb = kern + b * W * W * 4;
  double acc[4] = {0.0, 0.0, 0.0, 0.0}, wacc[4] = {0.0, 0.0, 0.0, 0.0};
  for (long long e = t; e < W * W; e += blockDim.x) {
    const int dx = (int)(e / W) - R, dy = (int)(e % W) - R;
    const long long px = ((dx + nx / 2) % nx + nx) % nx, py = ((dy + ny / 2) % ny + ny) % ny;
    for (int c = 0; c < 4; ++c) {
      const double val = r[(px * ny + py) * 4 + c];
      kb[e * 4 + c] = val;
      wacc[c] += val;
    }
  }
  for (long long v = t; v < nv; v += blockDim.x)
    for (int c = 0; c < 4; ++c) acc[c] += r[v * 4 + c];
  for (int pass = 0; pass < 2; ++pass) {
    double* src = pass ? wacc : acc;
    for (int c = 0; c < 4; ++c) red[c][t] = src[c];
    __syncthreads();
    for (int h = blockDim.x / 2; h > 0; h >>= 1) {
      if (t < h)
        for (int c = 0; c < 4; ++c) red[c][t] += red[c][t + h];
      __syncthreads();
    }
    if (t == 0)
      for (int c = 0; c < 4; ++c) src[c] = red[c][0];
    __syncthreads();
  }
  if (t == 0)
    for (int c = 0; c < 4; ++c) miss[b * 4 + c] = acc[c] / (double)nv - wacc[c] / (double)nv;
}

// Parallel inclusive FP64 scan (fast selection mode): per-block scans of
// 1024 rates, an exclusive scan of the block totals, and the offsets.  The
// running sums differ from the sequential chain by rounding only.
__global__ void scan_block_kernel(const double* __restrict__ r, long long n, double* __restrict__ prefix,
                                  double* __restrict__ bsum) {
  __shared__ double ws[32];
  const long long base = (long long)blockIdx.x * 1024;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  double v[4];
  double acc = 0.0;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const long long i = base + threadIdx.x * 4 + q;
    acc += (i < n) ? r[i] : 0.0;
    v[q] = acc;
  }
  double x = acc;
  for (int o = 1; o < 32; o <<= 1) { double y = __shfl_up_sync(0xffffffffu, x, o); if (lane >= o) x += y; }
  if (lane == 31) ws[wid] = x;
  __syncthreads();
  if (wid == 0) {
    double w = lane < (int)(blockDim.x >> 5) ? ws[lane] : 0.0;
    for (int o = 1; o < 32; o <<= 1) { double y = __shfl_up_sync(0xffffffffu, w, o); if (lane >= o) w += y; }
    ws[lane] = w;
  }
  __syncthreads();
  const double off = (x - acc) + (wid > 0 ? ws[wid - 1] : 0.0);
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const long long i = base + threadIdx.x * 4 + q;
    if (i < n) prefix[i] = off + v[q];
  }
  if (threadIdx.x == blockDim.x - 1) bsum[blockIdx.x] = off + acc;
}

__global__ void scan_bsum_kernel(double* bsum, int nb, long long n, double* d_total) {
  // single-thread exclusive scan of the (few hundred) block totals
  if (threadIdx.x != 0) return;
  double run = 0.0;
  for (int b = 0; b < nb; ++b) { const double t = bsum[b]; bsum[b] = run; run += t; }
  *d_total = n > 0 ? run : 0.0;
}

__global__ void scan_add_kernel(double* prefix, long long n, const double* bsum) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) prefix[i] += bsum[i / 1024];
}

}  // namespace mgk

using namespace mgk;

static int blocks_for(long long n, int bs) { return (int)((n + bs - 1) / bs); }

extern "C" int mgk_kmc2d_barrier(int nx, int ny, int M, double* Q, const double* Q0, const double* sig,
                                 const double* catalog, double volume, const double* soft_prop,
                                 const double* last_event_time, double current_time,
                                 const double* prev_strain_dir, double softening_cap, int scheme, double tau,
                                 mgk_stream_t stream) {
  MGK_REQUIRE(nx > 0 && ny > 0 && M > 0, "mgk_kmc2d_barrier: bad shape");
  MGK_REQUIRE(Q && Q0 && sig && catalog && soft_prop && last_event_time, "mgk_kmc2d_barrier: null argument");
  MGK_REQUIRE(scheme == 0 || (scheme == 1 && prev_strain_dir), "mgk_kmc2d_barrier: bad scheme");
  const long long nvox = (long long)nx * ny;
  barrier_kernel<2, 2><<<blocks_for(nvox * M, 256), 256, 0, (cudaStream_t)stream>>>(
      nvox, M, Q, Q0, sig, catalog, volume, soft_prop, last_event_time, current_time, prev_strain_dir,
      softening_cap, scheme, tau);
  MGK_CUDA(cudaGetLastError());
  return MGK_OK;
}

extern "C" int mgk_kmc2d_barrier_total(int nx, int ny, int M, double* Q, const double* Q0, const double* sig,
                                       const double* catalog, double volume, const double* soft_prop,
                                       const double* last_event_time, double current_time,
                                       const double* prev_strain_dir, double softening_cap, int scheme, double tau,
                                       double rate_volume, const double* temperature, double temperature_scalar,
                                       double nu0, double* d_total, void* work, mgk_stream_t stream) {
  MGK_REQUIRE(nx > 0 && ny > 0 && M > 0, "mgk_kmc2d_barrier_total: bad shape");
  MGK_REQUIRE(Q && Q0 && sig && catalog && soft_prop && last_event_time && d_total && work,
              "mgk_kmc2d_barrier_total: null argument");
  MGK_REQUIRE(scheme == 0 || (scheme == 1 && prev_strain_dir), "mgk_kmc2d_barrier_total: bad scheme");
  const long long nvox = (long long)nx * ny, n = nvox * M;
  // partials fit the scan work buffer: at most n / 1024 + 1 CTAs
  const int nb = (int)std::max(1LL, std::min(1184LL, n / 1024));
  const double vnu = rate_volume * nu0;  // host product, as in mgk_kmc2d_rates
  cudaStream_t s = (cudaStream_t)stream;
  double* partials = reinterpret_cast<double*>(work);
  barrier_total_kernel<2, 2><<<nb, 256, 0, s>>>(nvox, M, Q, Q0, sig, catalog, volume, soft_prop, last_event_time,
                                                current_time, prev_strain_dir, softening_cap, scheme, tau,
                                                temperature, temperature_scalar, vnu, partials);
  partials_total_kernel<<<1, 256, 0, s>>>(partials, nb, d_total);
  MGK_CUDA(cudaGetLastError());
  return MGK_OK;
}

extern "C" int64_t mgk_kmc_rates_work_bytes(int64_t n_modes) {
  return (int64_t)sizeof(int) * ((n_modes + 255) / 256 + 1);
}

static int kmc_rates_impl(long long nvox, int M, const double* Q, double volume, const double* T, double Ts,
                          double nu0, int cascade_mode, double* rates, int64_t* indices, double* prefix,
                          int64_t* d_count, double* d_total, void* work, cudaStream_t s) {
  const long long n = nvox * M;
  const double vnu = volume * nu0;  // host product, same rounding as (volume * nu0) in the reference
  if (!cascade_mode) {
    rates_full_kernel<<<blocks_for(n, 256), 256, 0, s>>>(nvox, M, Q, vnu, T, Ts, rates, (long long*)indices,
                                                         (long long*)d_count);
    MGK_CUDA(cudaGetLastError());
    int rc = launch_exact_prefix(rates, n, nullptr, prefix, d_total, s);
    if (rc) return rc;
  } else {
    MGK_REQUIRE(work != nullptr, "mgk_kmc2d_rates: cascade mode needs the work buffer");
    const int nb = blocks_for(n, 256);
    int* bcount = reinterpret_cast<int*>(work);
    rates_count_kernel<<<nb, 256, 0, s>>>(n, Q, bcount);
    MGK_CUDA(cudaGetLastError());
    scan_counts_kernel<<<1, 1024, 0, s>>>(nb, bcount, (long long*)d_count);
    MGK_CUDA(cudaGetLastError());
    rates_scatter_kernel<<<nb, 256, 0, s>>>(nvox, M, Q, vnu, T, Ts, bcount, rates, (long long*)indices);
    MGK_CUDA(cudaGetLastError());
    int rc = launch_exact_prefix(rates, n, (const long long*)d_count, prefix, d_total, s);
    if (rc) return rc;
  }
  return MGK_OK;
}

extern "C" int mgk_kmc2d_rates(int nx, int ny, int M, const double* Q, double volume, const double* temperature,
                               double temperature_scalar, double nu0, int cascade_mode, double* rates,
                               int64_t* indices, double* prefix, int64_t* d_count, double* d_total, void* work,
                               mgk_stream_t stream) {
  MGK_REQUIRE(nx > 0 && ny > 0 && M > 0, "mgk_kmc2d_rates: bad shape");
  MGK_REQUIRE(Q && rates && indices && prefix && d_count && d_total, "mgk_kmc2d_rates: null argument");
  return kmc_rates_impl((long long)nx * ny, M, Q, volume, temperature, temperature_scalar, nu0, cascade_mode, rates,
                        indices, prefix, d_count, d_total, work, (cudaStream_t)stream);
}

__global__ void set_count_kernel(long long* d_count, long long n) { *d_count = n; }

extern "C" int mgk_kmc_prefix(const double* rates, int64_t n, double* prefix, int64_t* d_count, double* d_total,
                              mgk_stream_t stream) {
  MGK_REQUIRE(n >= 0 && (n == 0 || (rates && prefix)) && d_count && d_total, "mgk_kmc_prefix: bad argument");
  cudaStream_t s = (cudaStream_t)stream;
  set_count_kernel<<<1, 1, 0, s>>>((long long*)d_count, (long long)n);
  MGK_CUDA(cudaGetLastError());
  return launch_exact_prefix(rates, n, nullptr, prefix, d_total, s);
}

extern "C" int mgk_kmc_select(const double* prefix, const int64_t* d_count, const double* d_total, double u,
                              int64_t* d_index, mgk_stream_t stream) {
  MGK_REQUIRE(prefix && d_count && d_total && d_index, "mgk_kmc_select: null argument");
  MGK_REQUIRE(u >= 0.0 && u < 1.0, "mgk_kmc_select: draw must be in [0, 1)");
  select_kernel<<<1, 1024, 0, (cudaStream_t)stream>>>(prefix, (const long long*)d_count, d_total, u,
                                                      (long long*)d_index);
  MGK_CUDA(cudaGetLastError());
  return MGK_OK;
}

extern "C" int mgk_kmc2d_flip(int nx, int ny, int M, double* eps_plastic, double* soft_prop, double* last_event_time,
                              const double* catalog, int x, int y, int m, double current_time, double jp, double jt,
                              double g_max, double jn_frac, mgk_stream_t stream) {
  MGK_REQUIRE(x >= 0 && x < nx && y >= 0 && y < ny && m >= 0 && m < M, "mgk_kmc2d_flip: index out of range");
  MGK_REQUIRE(eps_plastic && soft_prop && last_event_time && catalog, "mgk_kmc2d_flip: null argument");
  flip2d_kernel<<<1, 1, 0, (cudaStream_t)stream>>>(nx, ny, M, eps_plastic, soft_prop, last_event_time, catalog, x, y,
                                                   m, current_time, jp, jt, g_max, jn_frac);
  MGK_CUDA(cudaGetLastError());
  return MGK_OK;
}

extern "C" int mgk_kmc3d_barrier(int nx, int ny, int nz, int M, double* Q, const double* Q0, const double* sig,
                                 const double* catalog, double volume, const double* soft_prop,
                                 const double* last_event_time, double current_time,
                                 const double* prev_strain_dir, double softening_cap, int scheme, double tau,
                                 mgk_stream_t stream) {
  MGK_REQUIRE(nx > 0 && ny > 0 && nz > 0 && M > 0, "mgk_kmc3d_barrier: bad shape");
  MGK_REQUIRE(Q && Q0 && sig && catalog && soft_prop && last_event_time, "mgk_kmc3d_barrier: null argument");
  MGK_REQUIRE(scheme == 0 || (scheme == 1 && prev_strain_dir), "mgk_kmc3d_barrier: bad scheme");
  const long long nvox = (long long)nx * ny * nz;
  barrier_kernel<3, 4><<<blocks_for(nvox * M, 256), 256, 0, (cudaStream_t)stream>>>(
      nvox, M, Q, Q0, sig, catalog, volume, soft_prop, last_event_time, current_time, prev_strain_dir,
      softening_cap, scheme, tau);
  MGK_CUDA(cudaGetLastError());
  return MGK_OK;
}

extern "C" int mgk_kmc3d_rates(int nx, int ny, int nz, int M, const double* Q, double volume,
                               const double* temperature, double temperature_scalar, double nu0, int cascade_mode,
                               double* rates, int64_t* indices, double* prefix, int64_t* d_count, double* d_total,
                               void* work, mgk_stream_t stream) {
  MGK_REQUIRE(nx > 0 && ny > 0 && nz > 0 && M > 0, "mgk_kmc3d_rates: bad shape");
  MGK_REQUIRE(Q && rates && indices && prefix && d_count && d_total, "mgk_kmc3d_rates: null argument");
  return kmc_rates_impl((long long)nx * ny * nz, M, Q, volume, temperature, temperature_scalar, nu0, cascade_mode,
                        rates, indices, prefix, d_count, d_total, work, (cudaStream_t)stream);
}

extern "C" int mgk_kmc3d_flip(int nx, int ny, int nz, int M, double* eps_plastic, double* soft_prop,
                              double* last_event_time, const double* catalog, int x, int y, int z, int m,
                              double current_time, double jp, double jt, double g_max, double jn_frac,
                              mgk_stream_t stream) {
  MGK_REQUIRE(x >= 0 && x < nx && y >= 0 && y < ny && z >= 0 && z < nz && m >= 0 && m < M,
              "mgk_kmc3d_flip: index out of range");
  MGK_REQUIRE(eps_plastic && soft_prop && last_event_time && catalog, "mgk_kmc3d_flip: null argument");
  flip3d_kernel<<<1, 1, 0, (cudaStream_t)stream>>>(nx, ny, nz, M, eps_plastic, soft_prop, last_event_time, catalog,
                                                   x, y, z, m, current_time, jp, jt, g_max, jn_frac);
  MGK_CUDA(cudaGetLastError());
  return MGK_OK;
}

extern "C" int mgk_kmc3d_event(int nx, int ny, int nz, int M, const int64_t* d_sel, const int64_t* indices,
                               double* eps_plastic, double* soft_prop, double* last_event_time, double* catalog,
                               double* Q0, double* prev_strain_dir, const double* new_catalog,
                               const double* new_q0, double current_time, double jp, double jt, double g_max,
                               double jn_frac, int64_t* d_xyzm, mgk_stream_t stream) {
  MGK_REQUIRE(nx > 0 && ny > 0 && nz > 0 && M > 0 && d_sel && eps_plastic && soft_prop && last_event_time &&
                  catalog && Q0 && prev_strain_dir,
              "mgk_kmc3d_event: bad argument");
  event3d_kernel<<<1, 1, 0, (cudaStream_t)stream>>>(nx, ny, nz, M, (const long long*)d_sel, (const long long*)indices,
                                                    eps_plastic, soft_prop, last_event_time, catalog, Q0,
                                                    prev_strain_dir, new_catalog, new_q0, current_time, jp, jt, g_max,
                                                    jn_frac, (long long*)d_xyzm);
  MGK_CUDA(cudaGetLastError());
  return MGK_OK;
}

extern "C" int mgk_kmc2d_event(int nx, int ny, int M, const int64_t* d_sel, const int64_t* indices,
                               double* eps_plastic, double* soft_prop, double* last_event_time, double* catalog,
                               double* Q0, double* prev_strain_dir, const double* new_catalog,
                               const double* new_q0, double current_time, double jp, double jt, double g_max,
                               double jn_frac, int64_t* d_xym, mgk_stream_t stream) {
  MGK_REQUIRE(nx > 0 && ny > 0 && M > 0 && d_sel && eps_plastic && soft_prop && last_event_time && catalog && Q0 &&
                  prev_strain_dir,
              "mgk_kmc2d_event: bad argument");
  event2d_kernel<<<1, 1, 0, (cudaStream_t)stream>>>(nx, ny, M, (const long long*)d_sel, (const long long*)indices,
                                                    eps_plastic, soft_prop, last_event_time, catalog, Q0,
                                                    prev_strain_dir, new_catalog, new_q0, current_time, jp, jt, g_max,
                                                    jn_frac, (long long*)d_xym);
  MGK_CUDA(cudaGetLastError());
  return MGK_OK;
}

extern "C" int mgk_kmc2d_patch_setup(int nx, int ny, int R, const double* r0, const double* r1, double* kernels,
                                     double* missing_mean, mgk_stream_t stream) {
  MGK_REQUIRE(nx > 0 && ny > 0 && R >= 0 && R <= 4096 && r0 && r1 && kernels && missing_mean,
              "mgk_kmc2d_patch_setup: bad argument");
  patch2d_setup_kernel<<<2, 256, 0, (cudaStream_t)stream>>>(nx, ny, R, r0, r1, kernels, missing_mean);
  MGK_CUDA(cudaGetLastError());
  return MGK_OK;
}

extern "C" int mgk_kmc2d_patch(int nx, int ny, int M, double* sig, const double* sig_unit, double unit_scale,
                               const double* kernels, const double* missing_mean, int R, const double* catalog,
                               const int64_t* d_sel, const int64_t* indices, mgk_stream_t stream) {
  MGK_REQUIRE(nx > 0 && ny > 0 && M > 0 && sig && R >= 0 && R <= 4096 &&
                  (!d_sel || (kernels && missing_mean && catalog)),
              "mgk_kmc2d_patch: bad argument");
  MGK_REQUIRE(((uintptr_t)sig & 15) == 0 && ((uintptr_t)sig_unit & 15) == 0,
              "mgk_kmc2d_patch: sig and sig_unit must be 16-byte aligned");
  const long long nv = (long long)nx * ny;
  patch2d_kernel<<<blocks_for(nv, 256), 256, 0, (cudaStream_t)stream>>>(
      nx, ny, M, sig, sig_unit, unit_scale, kernels, missing_mean, R, catalog, (const long long*)d_sel,
      (const long long*)indices);
  MGK_CUDA(cudaGetLastError());
  return MGK_OK;
}

extern "C" int64_t mgk_kmc_scan_work_bytes(int64_t n) { return (int64_t)sizeof(double) * ((n + 1023) / 1024 + 1); }

extern "C" int mgk_kmc_prefix_fast(const double* rates, int64_t n, double* prefix, int64_t* d_count, double* d_total,
                                   void* work, mgk_stream_t stream) {
  MGK_REQUIRE(n >= 0 && (n == 0 || (rates && prefix)) && d_count && d_total && work, "mgk_kmc_prefix_fast: bad argument");
  cudaStream_t s = (cudaStream_t)stream;
  const int nb = (int)((n + 1023) / 1024);
  double* bsum = reinterpret_cast<double*>(work);
  set_count_kernel<<<1, 1, 0, s>>>((long long*)d_count, (long long)n);
  if (nb > 0) {
    scan_block_kernel<<<nb, 256, 0, s>>>(rates, n, prefix, bsum);
    scan_bsum_kernel<<<1, 32, 0, s>>>(bsum, nb, n, d_total);
    scan_add_kernel<<<(int)((n + 255) / 256), 256, 0, s>>>(prefix, n, bsum);
  } else {
    scan_bsum_kernel<<<1, 32, 0, s>>>(bsum, 0, 0, d_total);
  }
  MGK_CUDA(cudaGetLastError());
  return MGK_OK;
}

extern "C" int mgk_kmc2d_rates_only(int nx, int ny, int M, const double* Q, double volume, const double* temperature,
                                    double temperature_scalar, double nu0, double* rates, mgk_stream_t stream) {
  MGK_REQUIRE(nx > 0 && ny > 0 && M > 0 && Q && rates, "mgk_kmc2d_rates_only: bad argument");
  const long long nvox = (long long)nx * ny, n = nvox * M;
  rates_full_kernel<<<blocks_for(n, 256), 256, 0, (cudaStream_t)stream>>>(nvox, M, Q, volume * nu0, temperature,
                                                                          temperature_scalar, rates, nullptr, nullptr);
  MGK_CUDA(cudaGetLastError());
  return MGK_OK;
}
