// Shared-memory Stockham FFT for line lengths n = 2^a 3^b (4 <= n <= 4096).
//
// A CTA transforms a batch of complex lines that sit in shared memory, one
// radix-R pass at a time (R in {2, 3, 4, 8}), ping-ponging between two shared
// buffers.  Pass p with stride Ns (product of the earlier radices) maps
// butterfly j of a line as
//     in  : a[j + r*n/R],            r = 0..R-1
//     tw  : W_{Ns*R}^{r*(j mod Ns)}  (table W_n^m = exp(-2 pi i m / n))
//     out : b[(j - j mod Ns)*R + j mod Ns + r*Ns]
// which leaves the result in natural order (self-sorting Stockham form).
// SIGN = -1 is the forward kernel exp(-2 pi i jk/n), SIGN = +1 the inverse
// (unnormalised).  Twiddles are read from a per-length table in global
// memory (L1-resident), computed once on the host in double precision.
#pragma once
#include "common.cuh"

namespace mgk {

struct FftLen {
  int n;
  int npass;
  int radix[8];
  const void* tw;  // n complex (T) entries, W_n^m
};

// host: radix schedule for n = 2^a 3^b; returns false if n is unsupported
bool fft_schedule(int n, FftLen* f);

template <int SIGN, typename C> __device__ __forceinline__ void dft2(C* v) {
  C a = v[0], b = v[1];
  v[0] = cadd(a, b);
  v[1] = csub(a, b);
}

template <int SIGN, typename C> __device__ __forceinline__ void dft4(C& v0, C& v1, C& v2, C& v3) {
  C a0 = cadd(v0, v2), a1 = csub(v0, v2);
  C a2 = cadd(v1, v3), a3 = cmul_i<SIGN>(csub(v1, v3));
  v0 = cadd(a0, a2);
  v2 = csub(a0, a2);
  v1 = cadd(a1, a3);
  v3 = csub(a1, a3);
}

template <int SIGN, typename C> __device__ __forceinline__ void dft8(C* v) {
  using R = decltype(C::x);
  const R h = R(0.70710678118654752440084436210485);
  dft4<SIGN>(v[0], v[2], v[4], v[6]);
  dft4<SIGN>(v[1], v[3], v[5], v[7]);
  // odd half times W8^k, W8 = exp(SIGN * 2 pi i / 8)
  C o1 = mk<C>(h * (v[3].x - SIGN * v[3].y), h * (v[3].y + SIGN * v[3].x));
  C o2 = cmul_i<SIGN>(v[5]);
  C o3 = mk<C>(-h * (v[7].x + SIGN * v[7].y), h * (SIGN * v[7].x - v[7].y));
  C e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6], o0 = v[1];
  v[0] = cadd(e0, o0); v[4] = csub(e0, o0);
  v[1] = cadd(e1, o1); v[5] = csub(e1, o1);
  v[2] = cadd(e2, o2); v[6] = csub(e2, o2);
  v[3] = cadd(e3, o3); v[7] = csub(e3, o3);
}

template <int SIGN, typename C> __device__ __forceinline__ void dft3(C* v) {
  using R = decltype(C::x);
  const R s3 = R(0.86602540378443864676372317075294);
  C s = cadd(v[1], v[2]);
  C d = csub(v[1], v[2]);
  C m = mk<C>(v[0].x - R(0.5) * s.x, v[0].y - R(0.5) * s.y);
  C t = cmul_i<SIGN>(mk<C>(s3 * d.x, s3 * d.y));
  v[0] = cadd(v[0], s);
  v[1] = cadd(m, t);
  v[2] = csub(m, t);
}

template <int R, int SIGN, typename C>
__device__ __forceinline__ void stockham_bfly(const C* __restrict__ src, C* __restrict__ dst, int j,
                                              int nb, int Ns, int twstride, const C* __restrict__ tw) {
  C v[R];
#pragma unroll
  for (int r = 0; r < R; ++r) v[r] = src[j + r * nb];
  const int k = j % Ns;
  if (k != 0) {
#pragma unroll
    for (int r = 1; r < R; ++r) {
      C w = __ldg(&tw[r * k * twstride]);
      if (SIGN > 0) w.y = -w.y;
      v[r] = cmul(v[r], w);
    }
  }
  if (R == 2) dft2<SIGN>(v);
  else if (R == 3) dft3<SIGN>(v);
  else if (R == 4) dft4<SIGN>(v[0], v[1], v[2], v[3]);
  else dft8<SIGN>(v);
  const int base = (j - k) * R + k;
#pragma unroll
  for (int r = 0; r < R; ++r) dst[base + r * Ns] = v[r];
}

// Transform `nlines` lines of length f.n held at a[line*ld ...]; b is scratch
// of the same shape.  All threads of the CTA must call.  Returns the buffer
// (a or b) that holds the result.  Ends with a __syncthreads().
template <int SIGN, typename C>
__device__ C* fft_lines(C* a, C* b, int nlines, int ld, const FftLen& f) {
  const C* tw = reinterpret_cast<const C*>(f.tw);
  const int n = f.n;
  int Ns = 1;
  for (int p = 0; p < f.npass; ++p) {
    const int R = f.radix[p];
    const int nb = n / R;
    const int total = nlines * nb;
    const int twstride = n / (Ns * R);
    for (int t = threadIdx.x; t < total; t += blockDim.x) {
      const int line = t / nb;
      const int j = t - line * nb;
      const C* s = a + line * ld;
      C* d = b + line * ld;
      switch (R) {
        case 8: stockham_bfly<8, SIGN>(s, d, j, nb, Ns, twstride, tw); break;
        case 4: stockham_bfly<4, SIGN>(s, d, j, nb, Ns, twstride, tw); break;
        case 3: stockham_bfly<3, SIGN>(s, d, j, nb, Ns, twstride, tw); break;
        default: stockham_bfly<2, SIGN>(s, d, j, nb, Ns, twstride, tw); break;
      }
    }
    __syncthreads();
    C* t = a; a = b; b = t;
    Ns *= R;
  }
  return a;
}

}  // namespace mgk

// ------------------------------------------------ compile-time lengths ---
// The same Stockham passes with the radix schedule, strides and divisors
// known at compile time (no integer division at run time), for the grid
// sides the benchmark workloads use; other lengths take fft_lines.
namespace mgk {

struct RadixList {
  int np;
  int r[8];
};

// same schedule as fft_schedule(): radix-3 passes first, then radix 8, 4, 2
constexpr RadixList make_sched(int n) {
  RadixList s{0, {0, 0, 0, 0, 0, 0, 0, 0}};
  int m = n, a = 0, b = 0;
  while (m % 3 == 0) { m /= 3; ++b; }
  while (m % 2 == 0) { m /= 2; ++a; }
  for (int i = 0; i < b; ++i) s.r[s.np++] = 3;
  int p8 = a / 3, rem = a % 3;
  if (rem == 1 && p8 >= 1) { p8 -= 1; rem = 4; }
  for (int i = 0; i < p8; ++i) s.r[s.np++] = 8;
  if (rem == 4) { s.r[s.np++] = 4; s.r[s.np++] = 4; }
  else if (rem == 2) s.r[s.np++] = 4;
  else if (rem == 1) s.r[s.np++] = 2;
  return s;
}

template <int N, int SIGN, int P, int NS, typename C>
__device__ __forceinline__ C* stat_pass(C* a, C* b, int nlines, int ld, const C* __restrict__ tw) {
  constexpr RadixList S = make_sched(N);
  if constexpr (P == S.np) {
    return a;
  } else {
    constexpr int R = S.r[P];
    constexpr int nb = N / R;
    constexpr int tws = N / (NS * R);
    const int total = nlines * nb;
    for (int t = threadIdx.x; t < total; t += blockDim.x) {
      const int line = t / nb;
      const int j = t - line * nb;
      const C* src = a + line * ld;
      C* dst = b + line * ld;
      C v[R];
#pragma unroll
      for (int r = 0; r < R; ++r) v[r] = src[j + r * nb];
      const int k = j % NS;
      if (NS > 1 && k != 0) {
#pragma unroll
        for (int r = 1; r < R; ++r) {
          C w = __ldg(&tw[r * k * tws]);
          if (SIGN > 0) w.y = -w.y;
          v[r] = cmul(v[r], w);
        }
      }
      if constexpr (R == 2) dft2<SIGN>(v);
      else if constexpr (R == 3) dft3<SIGN>(v);
      else if constexpr (R == 4) dft4<SIGN>(v[0], v[1], v[2], v[3]);
      else dft8<SIGN>(v);
      const int base = (j - k) * R + k;
#pragma unroll
      for (int r = 0; r < R; ++r) dst[base + r * NS] = v[r];
    }
    __syncthreads();
    return stat_pass<N, SIGN, P + 1, NS * R>(b, a, nlines, ld, tw);
  }
}

// FFT of nlines lines: compile-time passes for the common lengths.
template <int SIGN, typename C>
__device__ __forceinline__ C* fft_any(C* a, C* b, int nlines, int ld, const FftLen& f) {
  const C* tw = reinterpret_cast<const C*>(f.tw);
  switch (f.n) {
    case 64: return stat_pass<64, SIGN, 0, 1>(a, b, nlines, ld, tw);
    case 96: return stat_pass<96, SIGN, 0, 1>(a, b, nlines, ld, tw);
    case 128: return stat_pass<128, SIGN, 0, 1>(a, b, nlines, ld, tw);
    case 192: return stat_pass<192, SIGN, 0, 1>(a, b, nlines, ld, tw);
    case 256: return stat_pass<256, SIGN, 0, 1>(a, b, nlines, ld, tw);
    case 384: return stat_pass<384, SIGN, 0, 1>(a, b, nlines, ld, tw);
    case 512: return stat_pass<512, SIGN, 0, 1>(a, b, nlines, ld, tw);
    case 768: return stat_pass<768, SIGN, 0, 1>(a, b, nlines, ld, tw);
    case 1024: return stat_pass<1024, SIGN, 0, 1>(a, b, nlines, ld, tw);
    default: return fft_lines<SIGN>(a, b, nlines, ld, f);
  }
}

}  // namespace mgk

// ------------------------------------------------------- warp-line FFTs ---
// One warp transforms L lines of a compile-time length N that sit in shared
// memory in a padded layout (one slot of slack per 128 bytes, so the strided
// stores of the early Stockham passes hit distinct banks).  Each pass reads
// all of a lane's butterfly inputs into registers, synchronises the warp,
// then writes the outputs in place: only the line's lanes synchronise between
// passes (__syncwarp, or a named barrier for two-warp lines), so
// warps of a CTA progress independently.
namespace mgk {

template <typename C> __device__ __forceinline__ int pidx(int i) {
  return sizeof(C) == 16 ? i + (i >> 3) : i + (i >> 4);
}
// elements per 128-byte padding period
template <typename C> constexpr int kPadPeriod = sizeof(C) == 16 ? 8 : 16;
// padded line length in elements, rounded up to 16 bytes
template <typename C> constexpr int padded_len(int n) {
  return sizeof(C) == 16 ? n + n / 8 + 1 : ((n + n / 16 + 1 + 1) & ~1);
}

// Synchronises the G lanes that share a line: the warp (G = 32) or two
// warps through named barrier `bid` (G = 64; ids 1.., 0 is __syncthreads).
template <int G> __device__ __forceinline__ void grp_sync(int bid) {
  if constexpr (G == 32) __syncwarp();
  else asm volatile("bar.sync %0, %1;" ::"r"(bid), "n"(G) : "memory");
}

template <int N, int SIGN, int L, int P, int NS, int G, typename C>
__device__ __forceinline__ void warp_pass(C* a, int stride, const C* __restrict__ tw, int lane, int bid) {
  constexpr RadixList S = make_sched(N);
  if constexpr (P < S.np) {
    constexpr int R = S.r[P];
    constexpr int nb = N / R;
    constexpr int U = (nb + G - 1) / G;
    constexpr int tws = N / (NS * R);
    C v[L][U][R];
#pragma unroll
    for (int l = 0; l < L; ++l)
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int j = lane + G * u;
        if (nb % G == 0 || j < nb) {
          if constexpr (nb % kPadPeriod<C> == 0) {
            // j + r*nb: the padding of r*nb is a constant, so one padded base
            const int pj = l * stride + pidx<C>(j);
#pragma unroll
            for (int r = 0; r < R; ++r) v[l][u][r] = a[pj + r * (nb + nb / kPadPeriod<C>)];
          } else {
#pragma unroll
            for (int r = 0; r < R; ++r) v[l][u][r] = a[l * stride + pidx<C>(j + r * nb)];
          }
        }
      }
    grp_sync<G>(bid);
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int j = lane + G * u;
      if (nb % G == 0 || j < nb) {
        const int k = j % NS;
        C w[R];
        if constexpr (NS > 1) {
#pragma unroll
          for (int r = 1; r < R; ++r) {
            w[r] = __ldg(&tw[r * k * tws]);
            if (SIGN > 0) w[r].y = -w[r].y;
          }
        }
        const int base = (j - k) * R + k;
#pragma unroll
        for (int l = 0; l < L; ++l) {
          C* x = v[l][u];
          if constexpr (NS > 1) {
#pragma unroll
            for (int r = 1; r < R; ++r) x[r] = cmul(x[r], w[r]);
          }
          if constexpr (R == 2) dft2<SIGN>(x);
          else if constexpr (R == 3) dft3<SIGN>(x);
          else if constexpr (R == 4) dft4<SIGN>(x[0], x[1], x[2], x[3]);
          else dft8<SIGN>(x);
          if constexpr (NS % kPadPeriod<C> == 0) {
            const int pb = l * stride + pidx<C>(base);
#pragma unroll
            for (int r = 0; r < R; ++r) a[pb + r * (NS + NS / kPadPeriod<C>)] = x[r];
          } else if constexpr (NS == 1 && kPadPeriod<C> % R == 0) {
            // base = j*R is a multiple of R, so base..base+R-1 share one padding block
            const int pb = l * stride + pidx<C>(base);
#pragma unroll
            for (int r = 0; r < R; ++r) a[pb + r] = x[r];
          } else {
#pragma unroll
            for (int r = 0; r < R; ++r) a[l * stride + pidx<C>(base + r * NS)] = x[r];
          }
        }
      }
    }
    grp_sync<G>(bid);
    warp_pass<N, SIGN, L, P + 1, NS * R, G>(a, stride, tw, lane, bid);
  }
}

// L lines at a, a + stride, ... (padded layout), transformed in place by the
// G lanes of the calling group (lane in [0, G)).  tw: the W_N^m table.
template <int N, int SIGN, int L, int G = 32, typename C>
__device__ __forceinline__ void warp_fft(C* a, int stride, const C* __restrict__ tw, int lane, int bid = 0) {
  warp_pass<N, SIGN, L, 0, 1, G>(a, stride, tw, lane, bid);
}

// line lengths with a compiled warp-line FFT
__host__ __device__ constexpr bool warp_fft_len(int n) {
  return n == 64 || n == 96 || n == 128 || n == 192 || n == 256 || n == 384 || n == 512 || n == 768 ||
         n == 1024;
}

// 16- or 8-byte asynchronous global -> shared copies (cp.async, completion
// tracked per thread with commit/wait groups)
__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)),
               "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_async8(void* dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)),
               "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
}
template <typename C> __device__ __forceinline__ void cp_async_elem(C* dst, const C* src) {
  if constexpr (sizeof(C) == 16) cp_async16(dst, src);
  else cp_async8(dst, src);
}

}  // namespace mgk
