// 2D small-strain Lippmann-Schwinger solver (FP64 / FP32 spectral path).
//
// Restates mgkmc/linear_elastic_simulator.py:12-88 (spectral_solver_2d):
//   tau = C:(eps - eps_p) - C0:eps;  eps_new = eps_bar - IFFT(Gamma0 : FFT(tau));
//   diff = ||eps_new - eps|| / (||eps|| + 1e-20); stop when diff < tol.
// with the Green operator of mgkmc/elasticity.py:20-53 evaluated on the fly
// from the wave vector (never materialised).
//
// HBM layout per replica (SoA planes of N = nx*ny doubles, C order):
//   mu, lam                 Lame fields (plane strain or plane stress lambda)
//   eps[3]                  xx, yy, symmetric xy of the current iterate
//   ep[3]                   xx, yy, symmetric xy of the eigenstrain
//   epa[2] (optional)       eps_p xy and yx when eps_p is not symmetric
//   spec[3]                 half spectrum, nx rows of ld = ny/2+1 complex
// The antisymmetric part of eps is uniform after the first iteration
// (Gamma0 returns symmetric tensors), so it is carried as one scalar.
//
// One iteration = two kernels:
//   row kernel  (one CTA per pair of x-rows): C2R along y of the previous
//               spectrum (two real rows packed as one complex line), update
//               eps = eps_bar + eps~, the diff/norm partial sums, then the
//               polarisation tau and the R2C along y of the next iteration;
//   column kernel (one CTA per tile of ky columns): complex FFT along x,
//               eps~^ = -Gamma0_sym(k) : tau^ / N, inverse FFT along x.
// So the spectral field crosses HBM once per direction per iteration.  The
// last CTA of each row kernel reduces the partial sums in a fixed order
// (deterministic), decides convergence on the device and drives the CUDA
// graph while-node that holds the loop.
//
// Nyquist handling: the reference takes .real of a complex ifft after
// multiplying by Gamma(q) whose sign pattern breaks Hermitian symmetry on
// Nyquist lines; .real of that equals the C2R of the operator averaged over
// q and its mirror, Gamma_sym(q) = (Gamma(q) + Gamma(S q))/2 with S flipping
// the Nyquist components, which is what the column kernel applies.  q uses
// numpy's fftfreq signs (-n/2 on an even axis's Nyquist line): where two axes
// sit on their Nyquist lines at once the average is Gamma(q) itself and the
// signs of the cross terms follow that convention.
#include <math.h>
#include <stddef.h>
#include <stdlib.h>

#include <vector>

#include "common.cuh"
#include "fft.cuh"

namespace mgk {

const void* twiddles(int n, int prec);

struct Ls2dRep {
  int nx, ny, nyh, ld;
  int row_base, row_items, col_base, col_items, tc;
  int has_epa;
  long long N;
  FftLen fx, fy;
  double* mu;
  double* lam;
  double* eps;   // 3 planes
  double* ep;    // 3 planes
  double* epa;   // 2 planes or null
  void* spec;    // 3 planes of nx*ld complex
};

struct Ls2dState {
  double mu0, lam0, Bc, inv2mu0;
  double ebar[3];
  double abar;
  double extra_d0, extra_n0;
  double tol;
  int max_iter;
  int iter;
  int done;
  int status;
  double diff;
  double means[4];  // warm-start means (xx, xy, yx, yy)
  double out_eps_mean[4];
  double out_sig_mean[4];
};

// --------------------------------------------------------------- helpers ---

// eps~^ = -Gamma0(n) : tau^ * scale for symmetric tau (2D), n a unit vector.
template <typename C, typename T>
__device__ __forceinline__ void gamma2d_apply(const C& txx, const C& tyy, const C& txy, T nx, T ny,
                                              T inv2mu0, T Bc, C& exx, C& eyy, C& exy) {
  C tnx = mk<C>(txx.x * nx + txy.x * ny, txx.y * nx + txy.y * ny);
  C tny = mk<C>(txy.x * nx + tyy.x * ny, txy.y * nx + tyy.y * ny);
  C ntn = mk<C>(tnx.x * nx + tny.x * ny, tnx.y * nx + tny.y * ny);
  const T a = T(2) * inv2mu0;
  exx = mk<C>(-(a * nx * tnx.x - Bc * nx * nx * ntn.x), -(a * nx * tnx.y - Bc * nx * nx * ntn.y));
  eyy = mk<C>(-(a * ny * tny.x - Bc * ny * ny * ntn.x), -(a * ny * tny.y - Bc * ny * ny * ntn.y));
  exy = mk<C>(-(inv2mu0 * (ny * tnx.x + nx * tny.x) - Bc * nx * ny * ntn.x),
              -(inv2mu0 * (ny * tnx.y + nx * tny.y) - Bc * nx * ny * ntn.y));
}

__device__ __forceinline__ int fftfreq(int k, int n) { return (k < (n + 1) / 2) ? k : k - n; }

// -------------------------------------------------------------- kernels ---

// Per-voxel material prep: mu, lambda from (E, nu) as in elasticity.py:3-10,
// eigenstrain planes, and per-CTA partial sums of E and nu for the means.
__global__ void ls2d_material_kernel(Ls2dRep* reps, int rep, const double* __restrict__ E,
                                     const double* __restrict__ nu, const double* __restrict__ epsp,
                                     int plane_mode, int set_moduli, double* partials) {
  __shared__ double red[32];
  Ls2dRep& R = reps[rep];
  const long long N = R.N;
  double sE = 0, sn = 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N;
       i += (long long)gridDim.x * blockDim.x) {
    if (set_moduli) {
      const double e = E[i], v = nu[i];
      const double mu = e / (2 * (1 + v));
      const double lam = plane_mode == MGK_PLANE_STRESS ? e * v / (1 - v * v)
                                                         : e * v / ((1 + v) * (1 - 2 * v));
      R.mu[i] = mu;
      R.lam[i] = lam;
      sE += e;
      sn += v;
    }
    double pxx = 0, pxy = 0, pyx = 0, pyy = 0;
    if (epsp) {
      pxx = epsp[4 * i + 0]; pxy = epsp[4 * i + 1]; pyx = epsp[4 * i + 2]; pyy = epsp[4 * i + 3];
    }
    R.ep[i] = pxx;
    R.ep[N + i] = pyy;
    R.ep[2 * N + i] = (pxy == pyx) ? pxy : 0.5 * (pxy + pyx);
    if (R.epa) {
      R.epa[i] = pxy;
      R.epa[N + i] = pyx;
    }
  }
  if (set_moduli) {
    double a = block_sum(sE, red);
    double b = block_sum(sn, red);
    if (threadIdx.x == 0) {
      partials[2 * blockIdx.x] = a;
      partials[2 * blockIdx.x + 1] = b;
    }
  }
}

// Reference medium from the means (linear_elastic_simulator.py:22-26).
__global__ void ls2d_medium_kernel(Ls2dRep* reps, Ls2dState* st, int rep, const double* partials,
                                   int nblocks, int plane_mode) {
  __shared__ double red[32];
  double a = 0, b = 0;
  for (int i = threadIdx.x; i < nblocks; i += blockDim.x) { a += partials[2 * i]; b += partials[2 * i + 1]; }
  a = block_sum(a, red);
  b = block_sum(b, red);
  if (threadIdx.x == 0) {
    const double N = (double)reps[rep].N;
    const double E = a / N, v = b / N;
    const double mu0 = E / (2 * (1 + v));
    const double lam0 = plane_mode == MGK_PLANE_STRESS ? E * v / (1 - v * v) : E * v / ((1 + v) * (1 - 2 * v));
    Ls2dState& S = st[rep];
    S.mu0 = mu0;
    S.lam0 = lam0;
    S.Bc = (lam0 + mu0) / (mu0 * (lam0 + 2 * mu0));
    S.inv2mu0 = 1.0 / (2 * mu0);
  }
}

// Means of a (nx,ny,2,2) field: per-CTA partials of the 4 components.
__global__ void aos4_partial_kernel(const double* __restrict__ f, long long N, double* partials) {
  __shared__ double red[32];
  double s[4] = {0, 0, 0, 0};
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N;
       i += (long long)gridDim.x * blockDim.x) {
    const double4 v = reinterpret_cast<const double4*>(f)[i];
    s[0] += v.x; s[1] += v.y; s[2] += v.z; s[3] += v.w;
  }
  for (int q = 0; q < 4; ++q) {
    double t = block_sum(s[q], red);
    if (threadIdx.x == 0) partials[4 * blockIdx.x + q] = t;
  }
}

// Sum K-wide partials of nblocks CTAs in a fixed order into out[K] (scaled).
__global__ void finalize_sums_kernel(const double* partials, int nblocks, int K, double scale, double* out) {
  __shared__ double red[32];
  for (int q = 0; q < K; ++q) {
    double a = 0;
    for (int i = threadIdx.x; i < nblocks; i += blockDim.x) a += partials[K * i + q];
    a = block_sum(a, red);
    if (threadIdx.x == 0) out[q] = a * scale;
  }
}

// Solve start: set eps_bar, tolerances and the initial field
// (linear_elastic_simulator.py:32-41); partial sums of the antisymmetric
// part's contribution to the first diff and norm.
__global__ void ls2d_begin_kernel(Ls2dRep* reps, Ls2dState* st, int rep, double e00, double e01,
                                  double e10, double e11, const double* __restrict__ eps_init,
                                  double tol, int max_iter, double* partials, unsigned int* counter) {
  __shared__ double red[32];
  Ls2dRep& R = reps[rep];
  Ls2dState& S = st[rep];
  const long long N = R.N;
  const double abar = 0.5 * (e01 - e10);
  const double sbar = (e01 == e10) ? e01 : 0.5 * (e01 + e10);
  double d2 = 0, n2 = 0;
  double m00 = 0, m01 = 0, m10 = 0, m11 = 0;
  if (eps_init) { m00 = S.means[0]; m01 = S.means[1]; m10 = S.means[2]; m11 = S.means[3]; }
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N;
       i += (long long)gridDim.x * blockDim.x) {
    if (eps_init) {
      const double4 v = reinterpret_cast<const double4*>(eps_init)[i];
      const double xx = v.x + (e00 - m00), xy = v.y + (e01 - m01);
      const double yx = v.z + (e10 - m10), yy = v.w + (e11 - m11);
      R.eps[i] = xx;
      R.eps[N + i] = yy;
      R.eps[2 * N + i] = (xy == yx) ? xy : 0.5 * (xy + yx);
      const double a0 = 0.5 * (xy - yx);
      d2 += 2 * (abar - a0) * (abar - a0);
      n2 += 2 * a0 * a0;
    } else {
      R.eps[i] = e00;
      R.eps[N + i] = e11;
      R.eps[2 * N + i] = sbar;
    }
  }
  if (eps_init) {
    d2 = block_sum(d2, red);
    n2 = block_sum(n2, red);
    if (threadIdx.x == 0) { partials[2 * blockIdx.x] = d2; partials[2 * blockIdx.x + 1] = n2; }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    counter[1] = 0;
    S.ebar[0] = e00;
    S.ebar[1] = e11;
    S.ebar[2] = sbar;
    S.abar = abar;
    S.tol = tol;
    S.max_iter = max_iter;
    S.iter = 0;
    S.done = max_iter <= 0 ? 1 : 0;
    S.status = MGK_OK;
    S.diff = 0;
    if (!eps_init) { S.extra_d0 = 0; S.extra_n0 = 2.0 * (double)N * abar * abar; }
  }
}

__global__ void ls2d_begin_finalize_kernel(Ls2dState* st, int rep, const double* partials, int nblocks) {
  __shared__ double red[32];
  double a = 0, b = 0;
  for (int i = threadIdx.x; i < nblocks; i += blockDim.x) { a += partials[2 * i]; b += partials[2 * i + 1]; }
  a = block_sum(a, red);
  b = block_sum(b, red);
  if (threadIdx.x == 0) { st[rep].extra_d0 = a; st[rep].extra_n0 = b; }
}

// Row kernel.  IN_SPEC: the previous iteration's spectrum is inverted and the
// field updated (with diff/norm); otherwise the field is read as is.
template <typename T, bool IN_SPEC>
__global__ void __launch_bounds__(256) ls2d_row_kernel(const Ls2dRep* __restrict__ reps, Ls2dState* st,
                                                      const int* __restrict__ row_map, double* partials,
                                                      unsigned int* counter, int nrep,
                                                      cudaGraphConditionalHandle cond, int use_cond,
                                                      int* any_active, int guard_cap) {
  using C = C_t<T>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ double red[32];
  __shared__ int s_last;
  const int item = blockIdx.x;
  const int r = row_map[item];
  const Ls2dRep& R = reps[r];
  Ls2dState& S = st[r];
  const bool active = S.done == 0;
  double d2 = 0, n2 = 0;
  if (active) {
    const int ny = R.ny, nyh = R.nyh, ld = R.ld, nx = R.nx;
    const long long N = R.N;
    const int x0 = 2 * (item - R.row_base);
    C* bufA = reinterpret_cast<C*>(smem_raw);
    C* bufB = bufA + 3 * ny;
    C* spec = reinterpret_cast<C*>(R.spec);
    const double mu0 = S.mu0, lam0 = S.lam0;
    const double eb0 = S.ebar[0], eb1 = S.ebar[1], eb2 = S.ebar[2];
    C* cur;  // holds the packed real rows (x0 real, x1 imag) of eps~ or nothing
    if (IN_SPEC) {
      for (int e = threadIdx.x; e < 3 * ny; e += blockDim.x) {
        const int c = e / ny, k = e - c * ny;
        const C* ra = spec + ((size_t)c * nx + x0) * ld;
        const C* rb = ra + ld;
        C z;
        if (2 * k <= ny) {
          C a = ra[k], b = rb[k];
          if (k == 0 || 2 * k == ny) { a.y = 0; b.y = 0; }
          z = mk<C>(a.x - b.y, a.y + b.x);
        } else {
          const C a = ra[ny - k], b = rb[ny - k];
          z = mk<C>(a.x + b.y, b.x - a.y);
        }
        bufA[c * ny + k] = z;
      }
      __syncthreads();
      cur = fft_lines<+1>(bufA, bufB, 3, ny, R.fy);
    }
    C* out = (IN_SPEC && cur == bufA) ? bufB : bufA;
    // update + tau (packed: real = row x0, imag = row x1)
    for (int y = threadIdx.x; y < ny; y += blockDim.x) {
      T tr[2][3];
      for (int h = 0; h < 2; ++h) {
        const long long i = (long long)(x0 + h) * ny + y;
        double e[3];
        for (int c = 0; c < 3; ++c) {
          const double old = R.eps[c * N + i];
          if (IN_SPEC) {
            const C z = cur[c * ny + y];
            const double et = h == 0 ? (double)z.x : (double)z.y;
            const double nw = (c == 0 ? eb0 : (c == 1 ? eb1 : eb2)) + et;
            const double dd = nw - old;
            const double w = c == 2 ? 2.0 : 1.0;
            d2 += w * dd * dd;
            n2 += w * old * old;
            R.eps[c * N + i] = nw;
            e[c] = nw;
          } else {
            e[c] = old;
          }
        }
        const double mu = R.mu[i], lam = R.lam[i];
        const double dxx = e[0] - R.ep[i], dyy = e[1] - R.ep[N + i], dxy = e[2] - R.ep[2 * N + i];
        const double trd = dxx + dyy, tre = e[0] + e[1];
        tr[h][0] = (T)((2 * mu * dxx + lam * trd) - (2 * mu0 * e[0] + lam0 * tre));
        tr[h][1] = (T)((2 * mu * dyy + lam * trd) - (2 * mu0 * e[1] + lam0 * tre));
        tr[h][2] = (T)(2 * mu * dxy - 2 * mu0 * e[2]);
      }
      for (int c = 0; c < 3; ++c) out[c * ny + y] = mk<C>(tr[0][c], tr[1][c]);
    }
    __syncthreads();
    C* scratch = (out == bufA) ? bufB : bufA;
    C* Z = fft_lines<-1>(out, scratch, 3, ny, R.fy);
    // unpack the two real rows' half spectra
    for (int e = threadIdx.x; e < 3 * nyh; e += blockDim.x) {
      const int c = e / nyh, k = e - c * nyh;
      const C z = Z[c * ny + k];
      const C w = Z[c * ny + (k == 0 ? 0 : ny - k)];
      C* ra = spec + ((size_t)c * nx + x0) * ld;
      ra[k] = mk<C>(T(0.5) * (z.x + w.x), T(0.5) * (z.y - w.y));
      ra[ld + k] = mk<C>(T(0.5) * (z.y + w.y), T(-0.5) * (z.x - w.x));
    }
  }
  if (!IN_SPEC) return;
  // partial sums -> fixed slot; the last CTA to finish reduces and decides
  d2 = block_sum(d2, red);
  n2 = block_sum(n2, red);
  if (threadIdx.x == 0) {
    partials[2 * item] = d2;
    partials[2 * item + 1] = n2;
    __threadfence();
    // wraps back to 0 on the last arrival, so the counter resets itself
    const unsigned int t = atomicInc(counter, gridDim.x - 1);
    s_last = (t == gridDim.x - 1);
    if (item == 0 && use_cond) {
      // independent bound on the number of loop bodies: counter[1] is reset by
      // the begin kernel; a loop that outlives every replica's cap is stopped
      const unsigned int g = atomicAdd(counter + 1, 1u);
      if (g > (unsigned int)guard_cap) cudaGraphSetConditional(cond, 0u);
    }
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  int any = 0;
  for (int q = 0; q < nrep; ++q) {
    Ls2dState& Q = st[q];
    if (Q.done) continue;
    const Ls2dRep& P = reps[q];
    double a = 0, b = 0;
    for (int i = threadIdx.x; i < P.row_items; i += blockDim.x) {
      a += __ldcg(&partials[2 * (P.row_base + i)]);
      b += __ldcg(&partials[2 * (P.row_base + i) + 1]);
    }
    a = block_sum(a, red);
    b = block_sum(b, red);
    if (threadIdx.x == 0) {
      if (Q.iter == 0) { a += Q.extra_d0; b += Q.extra_n0; }
      else { b += 2.0 * (double)P.N * Q.abar * Q.abar; }
      const double diff = sqrt(a) / (sqrt(b) + 1e-20);
      Q.diff = diff;
      Q.iter += 1;
      if (!isfinite(diff)) { Q.done = 1; Q.status = MGK_NONFINITE; }
      else if (diff < Q.tol) { Q.done = 1; Q.status = MGK_OK; }
      else if (Q.iter >= Q.max_iter) { Q.done = 1; Q.status = MGK_NOT_CONVERGED; }
      else any = 1;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    *any_active = any;
    if (use_cond) {
      const bool over = atomicAdd(counter + 1, 0u) > (unsigned int)guard_cap;
      cudaGraphSetConditional(cond, (any && !over) ? 1u : 0u);
    }
  }
}

// Column kernel: FFT along x, Gamma0_sym, inverse FFT along x, for a tile of
// tc consecutive ky columns and all three components.
template <typename T>
__global__ void __launch_bounds__(256) ls2d_col_kernel(const Ls2dRep* __restrict__ reps,
                                                      const Ls2dState* __restrict__ st,
                                                      const int* __restrict__ col_map) {
  using C = C_t<T>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int item = blockIdx.x;
  const int r = col_map[item];
  const Ls2dRep& R = reps[r];
  const Ls2dState& S = st[r];
  if (S.done) return;
  const int nx = R.nx, ny = R.ny, nyh = R.nyh, ld = R.ld, tc = R.tc;
  const int ky0 = (item - R.col_base) * tc;
  const int tcw = min(tc, nyh - ky0);
  C* bufA = reinterpret_cast<C*>(smem_raw);
  C* bufB = bufA + 3 * tc * nx;
  C* spec = reinterpret_cast<C*>(R.spec);
  const int tot = 3 * tcw * nx;
  for (int e = threadIdx.x; e < tot; e += blockDim.x) {
    const int c = e / (tcw * nx);
    const int rem = e - c * tcw * nx;
    const int x = rem / tcw, t = rem - x * tcw;
    bufA[(c * tc + t) * nx + x] = spec[((size_t)c * nx + x) * ld + ky0 + t];
  }
  __syncthreads();
  // lines: (c * tc + t), only t < tcw are meaningful; transform all 3*tc lines
  C* F = fft_lines<-1>(bufA, bufB, 3 * tc, nx, R.fx);
  const T inv2mu0 = (T)S.inv2mu0, Bc = (T)S.Bc;
  const double scale = 1.0 / ((double)nx * (double)ny);
  for (int e = threadIdx.x; e < tcw * nx; e += blockDim.x) {
    const int t = e / nx, kx = e - t * nx;
    const int ky = ky0 + t;
    C* pxx = &F[(0 * tc + t) * nx + kx];
    C* pyy = &F[(1 * tc + t) * nx + kx];
    C* pxy = &F[(2 * tc + t) * nx + kx];
    if (kx == 0 && ky == 0) {
      *pxx = mk<C>(T(0), T(0)); *pyy = *pxx; *pxy = *pxx;
      continue;
    }
    // fftfreq signs matter where several axes sit on their Nyquist line
    const double ux = (double)fftfreq(kx, nx) / nx, uy = (double)fftfreq(ky, ny) / ny;
    const double inv = 1.0 / sqrt(ux * ux + uy * uy);
    const T nxv = (T)(ux * inv), nyv = (T)(uy * inv);
    C txx = *pxx, tyy = *pyy, txy = *pxy;
    C exx, eyy, exy;
    gamma2d_apply(txx, tyy, txy, nxv, nyv, inv2mu0, Bc, exx, eyy, exy);
    const bool nyq = ((nx & 1) == 0 && 2 * kx == nx) || ((ny & 1) == 0 && 2 * ky == ny);
    if (nyq) {
      const T sx = ((nx & 1) == 0 && 2 * kx == nx) ? -nxv : nxv;
      const T sy = ((ny & 1) == 0 && 2 * ky == ny) ? -nyv : nyv;
      C fxx, fyy, fxy;
      gamma2d_apply(txx, tyy, txy, sx, sy, inv2mu0, Bc, fxx, fyy, fxy);
      exx = mk<C>(T(0.5) * (exx.x + fxx.x), T(0.5) * (exx.y + fxx.y));
      eyy = mk<C>(T(0.5) * (eyy.x + fyy.x), T(0.5) * (eyy.y + fyy.y));
      exy = mk<C>(T(0.5) * (exy.x + fxy.x), T(0.5) * (exy.y + fxy.y));
    }
    const T sc = (T)scale;
    *pxx = mk<C>(exx.x * sc, exx.y * sc);
    *pyy = mk<C>(eyy.x * sc, eyy.y * sc);
    *pxy = mk<C>(exy.x * sc, exy.y * sc);
  }
  __syncthreads();
  C* G = (F == bufA) ? bufB : bufA;
  C* Rz = fft_lines<+1>(F, G, 3 * tc, nx, R.fx);
  for (int e = threadIdx.x; e < tot; e += blockDim.x) {
    const int c = e / (tcw * nx);
    const int rem = e - c * tcw * nx;
    const int x = rem / tcw, t = rem - x * tcw;
    spec[((size_t)c * nx + x) * ld + ky0 + t] = Rz[(c * tc + t) * nx + x];
  }
}

// Outputs in the reference layout: eps, sig (nx,ny,2,2) and partial sums of
// their components for the means (linear_elastic_simulator.py:83-88).
__global__ void ls2d_output_kernel(const Ls2dRep* reps, const Ls2dState* st, int rep, double* eps_out,
                                   double* sig_out, double* partials) {
  __shared__ double red[32];
  const Ls2dRep& R = reps[rep];
  const Ls2dState& S = st[rep];
  const long long N = R.N;
  const double abar = S.abar;
  double s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N;
       i += (long long)gridDim.x * blockDim.x) {
    const double sxy = R.eps[2 * N + i];
    const double exx = R.eps[i], eyy = R.eps[N + i];
    const double exy = abar == 0 ? sxy : sxy + abar;
    const double eyx = abar == 0 ? sxy : sxy - abar;
    double pxx = R.ep[i], pyy = R.ep[N + i], pxy, pyx;
    if (R.epa) { pxy = R.epa[i]; pyx = R.epa[N + i]; }
    else { pxy = R.ep[2 * N + i]; pyx = pxy; }
    const double mu = R.mu[i], lam = R.lam[i];
    const double dxx = exx - pxx, dxy = exy - pxy, dyx = eyx - pyx, dyy = eyy - pyy;
    const double tr = dxx + dyy;
    const double sxx = 2 * mu * dxx + lam * tr, syy = 2 * mu * dyy + lam * tr;
    const double sxy2 = 2 * mu * dxy, syx2 = 2 * mu * dyx;
    if (eps_out) reinterpret_cast<double4*>(eps_out)[i] = make_double4(exx, exy, eyx, eyy);
    if (sig_out) reinterpret_cast<double4*>(sig_out)[i] = make_double4(sxx, sxy2, syx2, syy);
    s[0] += exx; s[1] += exy; s[2] += eyx; s[3] += eyy;
    s[4] += sxx; s[5] += sxy2; s[6] += syx2; s[7] += syy;
  }
  for (int q = 0; q < 8; ++q) {
    double t = block_sum(s[q], red);
    if (threadIdx.x == 0) partials[8 * blockIdx.x + q] = t;
  }
}

}  // namespace mgk

// ================================================================== plan ===
using namespace mgk;

struct mgk_ls2d_plan {
  int nx, ny, nyh, ld, tc, plane_mode, prec;
  long long N;
  int row_items, col_items;
  size_t row_smem, col_smem;
  Ls2dRep h_rep;
  Ls2dRep* d_rep = nullptr;
  Ls2dState* d_st = nullptr;
  int* d_rowmap = nullptr;
  int* d_colmap = nullptr;
  double* d_part = nullptr;
  int n_part = 0;
  unsigned int* d_counter = nullptr;
  int* d_any = nullptr;
  double* d_fields = nullptr;
  void* d_spec = nullptr;
  bool has_material = false;
  bool has_epa = false;
  // loop graph
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int graph_mode = -1;  // -1 untried, 1 while-node graph, 0 host loop
  int guard_cap = 0;     // loop-body bound baked into the graph (max_iter of the build + 2)
  Ls2dState* h_state = nullptr;  // pinned
  int* h_any = nullptr;          // pinned
};

static int grid_for(long long N) {
  long long b = (N + 255) / 256;
  if (b > 2048) b = 2048;
  if (b < 1) b = 1;
  return (int)b;
}

template <typename T>
static int ls2d_configure(mgk_ls2d_t p) {
  using C = C_t<T>;
  p->row_smem = 2 * 3 * (size_t)p->ny * sizeof(C);
  p->col_smem = 2 * 3 * (size_t)p->tc * p->nx * sizeof(C);
  MGK_CUDA(cudaFuncSetAttribute(ls2d_row_kernel<T, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)p->row_smem));
  MGK_CUDA(cudaFuncSetAttribute(ls2d_row_kernel<T, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)p->row_smem));
  MGK_CUDA(cudaFuncSetAttribute(ls2d_col_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)p->col_smem));
  return MGK_OK;
}

extern "C" int mgk_ls2d_destroy(mgk_ls2d_t p) {
  if (!p) return MGK_OK;
  if (p->exec) cudaGraphExecDestroy(p->exec);
  if (p->graph) cudaGraphDestroy(p->graph);
  cudaFree(p->d_rep);
  cudaFree(p->d_st);
  cudaFree(p->d_rowmap);
  cudaFree(p->d_colmap);
  cudaFree(p->d_part);
  cudaFree(p->d_counter);
  cudaFree(p->d_any);
  cudaFree(p->d_fields);
  cudaFree(p->d_spec);
  if (p->h_state) cudaFreeHost(p->h_state);
  if (p->h_any) cudaFreeHost(p->h_any);
  delete p;
  return MGK_OK;
}

extern "C" int mgk_ls2d_create(int nx, int ny, int plane_mode, int precision, mgk_ls2d_t* out) {
  MGK_REQUIRE(out != nullptr, "mgk_ls2d_create: null output handle");
  *out = nullptr;
  MGK_REQUIRE(plane_mode == MGK_PLANE_STRAIN || plane_mode == MGK_PLANE_STRESS,
              "mgk_ls2d_create: plane_mode must be 0 (strain) or 1 (stress)");
  MGK_REQUIRE(precision == MGK_FP64 || precision == MGK_FP32, "mgk_ls2d_create: bad precision");
  FftLen fx, fy;
  MGK_REQUIRE(fft_schedule(nx, &fx) && fft_schedule(ny, &fy),
              "mgk_ls2d_create: grid %dx%d unsupported (each side must be 2^a 3^b, even, 4..4096)", nx, ny);
  mgk_ls2d_t p = new mgk_ls2d_plan();
  p->nx = nx; p->ny = ny; p->nyh = ny / 2 + 1; p->ld = p->nyh;
  p->plane_mode = plane_mode; p->prec = precision;
  p->N = (long long)nx * ny;
  const size_t csz = precision == MGK_FP64 ? sizeof(double2) : sizeof(float2);
  // columns per CTA: largest power of two <= 8 whose tile fits in ~200 KB
  int tc = 8;
  while (tc > 1 && 2 * 3 * (size_t)tc * nx * csz > 200 * 1024) tc >>= 1;
  p->tc = tc;
  MGK_REQUIRE(2 * 3 * (size_t)tc * nx * csz <= 220 * 1024 && 2 * 3 * (size_t)ny * csz <= 220 * 1024,
              "mgk_ls2d_create: grid too large for the shared-memory FFT");
  p->row_items = nx / 2;
  p->col_items = (p->nyh + tc - 1) / tc;
  int st = precision == MGK_FP64 ? ls2d_configure<double>(p) : ls2d_configure<float>(p);
  if (st != MGK_OK) { delete p; return st; }
  const long long N = p->N;
  const size_t spec_bytes = 3 * (size_t)nx * p->ld * csz;
  auto fail = [&](int s) { mgk_ls2d_destroy(p); return s; };
  if (cudaMalloc(&p->d_fields, sizeof(double) * N * 13) != cudaSuccess) return fail(MGK_OOM);
  if (cudaMalloc(&p->d_spec, spec_bytes) != cudaSuccess) return fail(MGK_OOM);
  if (cudaMalloc(&p->d_rep, sizeof(Ls2dRep)) != cudaSuccess) return fail(MGK_OOM);
  if (cudaMalloc(&p->d_st, sizeof(Ls2dState)) != cudaSuccess) return fail(MGK_OOM);
  if (cudaMalloc(&p->d_rowmap, sizeof(int) * p->row_items) != cudaSuccess) return fail(MGK_OOM);
  if (cudaMalloc(&p->d_colmap, sizeof(int) * p->col_items) != cudaSuccess) return fail(MGK_OOM);
  p->n_part = 2048;
  if (p->n_part < p->row_items) p->n_part = p->row_items;
  if (cudaMalloc(&p->d_part, sizeof(double) * 8 * p->n_part) != cudaSuccess) return fail(MGK_OOM);
  if (cudaMalloc(&p->d_counter, 2 * sizeof(unsigned int)) != cudaSuccess) return fail(MGK_OOM);
  if (cudaMalloc(&p->d_any, sizeof(int)) != cudaSuccess) return fail(MGK_OOM);
  if (cudaMallocHost(&p->h_state, sizeof(Ls2dState)) != cudaSuccess) return fail(MGK_OOM);
  if (cudaMemset(p->d_counter, 0, 2 * sizeof(unsigned int)) != cudaSuccess) return fail(MGK_CUDA_ERROR);
  if (cudaMallocHost(&p->h_any, sizeof(int)) != cudaSuccess) return fail(MGK_OOM);
  if (cudaMemset(p->d_st, 0, sizeof(Ls2dState)) != cudaSuccess) return fail(MGK_CUDA_ERROR);
  fx.tw = twiddles(nx, precision);
  fy.tw = twiddles(ny, precision);
  if (!fx.tw || !fy.tw) return fail(MGK_OOM);
  Ls2dRep& R = p->h_rep;
  memset(&R, 0, sizeof(R));
  R.nx = nx; R.ny = ny; R.nyh = p->nyh; R.ld = p->ld;
  R.row_base = 0; R.row_items = p->row_items; R.col_base = 0; R.col_items = p->col_items; R.tc = tc;
  R.N = N; R.fx = fx; R.fy = fy;
  double* f = p->d_fields;
  R.mu = f; R.lam = f + N; R.eps = f + 2 * N; R.ep = f + 5 * N; R.epa = nullptr;
  R.spec = p->d_spec;
  std::vector<int> rm(p->row_items, 0), cm(p->col_items, 0);
  if (cudaMemcpy(p->d_rowmap, rm.data(), sizeof(int) * rm.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(p->d_colmap, cm.data(), sizeof(int) * cm.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(p->d_rep, &R, sizeof(R), cudaMemcpyHostToDevice) != cudaSuccess)
    return fail(MGK_CUDA_ERROR);
  *out = p;
  return MGK_OK;
}

static int ls2d_upload_rep(mgk_ls2d_t p, cudaStream_t s) {
  MGK_CUDA(cudaMemcpyAsync(p->d_rep, &p->h_rep, sizeof(Ls2dRep), cudaMemcpyHostToDevice, s));
  return MGK_OK;
}

static int ls2d_set_fields(mgk_ls2d_t p, const double* E, const double* nu, const double* epsp,
                           int set_moduli, cudaStream_t s) {
  // eigenstrain asymmetry must be known before the kernel: scan on the host
  // side is impossible for device data, so keep the xy/yx planes whenever a
  // field is given and let the kernel store both (cheap, 2 extra planes).
  const bool want_epa = epsp != nullptr;
  if (want_epa != (p->h_rep.epa != nullptr)) {
    p->h_rep.epa = want_epa ? p->d_fields + 8 * p->N : nullptr;
    p->h_rep.has_epa = want_epa;
    int st = ls2d_upload_rep(p, s);
    if (st) return st;
  }
  const int grid = grid_for(p->N);
  ls2d_material_kernel<<<grid, 256, 0, s>>>(p->d_rep, 0, E, nu, epsp, p->plane_mode, set_moduli, p->d_part);
  MGK_CUDA(cudaGetLastError());
  if (set_moduli) {
    ls2d_medium_kernel<<<1, 256, 0, s>>>(p->d_rep, p->d_st, 0, p->d_part, grid, p->plane_mode);
    MGK_CUDA(cudaGetLastError());
  }
  return MGK_OK;
}

extern "C" int mgk_ls2d_set_material(mgk_ls2d_t p, const double* E, const double* nu, const double* epsp,
                                     mgk_stream_t stream) {
  MGK_REQUIRE(p && E && nu, "mgk_ls2d_set_material: null argument");
  int st = ls2d_set_fields(p, E, nu, epsp, 1, (cudaStream_t)stream);
  if (st == MGK_OK) p->has_material = true;
  return st;
}

extern "C" int mgk_ls2d_set_eigenstrain(mgk_ls2d_t p, const double* epsp, mgk_stream_t stream) {
  MGK_REQUIRE(p && p->has_material, "mgk_ls2d_set_eigenstrain: plan has no material");
  return ls2d_set_fields(p, nullptr, nullptr, epsp, 0, (cudaStream_t)stream);
}

template <typename T>
static int ls2d_launch_body(mgk_ls2d_t p, cudaStream_t s, int use_cond, cudaGraphConditionalHandle h) {
  ls2d_col_kernel<T><<<p->col_items, 256, p->col_smem, s>>>(p->d_rep, p->d_st, p->d_colmap);
  MGK_CUDA(cudaGetLastError());
  ls2d_row_kernel<T, true><<<p->row_items, 256, p->row_smem, s>>>(
      p->d_rep, p->d_st, p->d_rowmap, p->d_part, p->d_counter, 1, h, use_cond, p->d_any, p->guard_cap);
  MGK_CUDA(cudaGetLastError());
  return MGK_OK;
}

template <typename T>
static int ls2d_build_graph(mgk_ls2d_t p) {
  cudaGraph_t g = nullptr;
  MGK_CUDA(cudaGraphCreate(&g, 0));
  cudaGraphConditionalHandle h;
  cudaError_t e = cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault);
  if (e != cudaSuccess) { cudaGraphDestroy(g); cudaGetLastError(); return MGK_CUDA_ERROR; }
  // cudaGraphNodeParams has no default constructor in C++: zeroed storage
  alignas(cudaGraphNodeParams) unsigned char cp_raw[sizeof(cudaGraphNodeParams)];
  memset(cp_raw, 0, sizeof(cp_raw));
  cudaGraphNodeParams& cp = *reinterpret_cast<cudaGraphNodeParams*>(cp_raw);
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = h;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  cudaGraphNode_t wnode;
  e = cudaGraphAddNode(&wnode, g, nullptr, 0, &cp);
  if (e != cudaSuccess) { cudaGraphDestroy(g); cudaGetLastError(); return MGK_CUDA_ERROR; }
  cudaGraph_t body = cp.conditional.phGraph_out[0];
  // kernel nodes of the body: column kernel -> row kernel
  cudaKernelNodeParams k1;
  memset(&k1, 0, sizeof(k1));
  void* a1[] = {&p->d_rep, &p->d_st, &p->d_colmap};
  k1.func = (void*)ls2d_col_kernel<T>;
  k1.gridDim = dim3(p->col_items);
  k1.blockDim = dim3(256);
  k1.sharedMemBytes = (unsigned)p->col_smem;
  k1.kernelParams = a1;
  cudaGraphNode_t n1, n2;
  e = cudaGraphAddKernelNode(&n1, body, nullptr, 0, &k1);
  if (e != cudaSuccess) { cudaGraphDestroy(g); cudaGetLastError(); return MGK_CUDA_ERROR; }
  int nrep = 1, use_cond = 1;
  cudaKernelNodeParams k2;
  memset(&k2, 0, sizeof(k2));
  void* a2[] = {&p->d_rep, &p->d_st, &p->d_rowmap, &p->d_part, &p->d_counter, &nrep, &h, &use_cond, &p->d_any,
                &p->guard_cap};
  k2.func = (void*)ls2d_row_kernel<T, true>;
  k2.gridDim = dim3(p->row_items);
  k2.blockDim = dim3(256);
  k2.sharedMemBytes = (unsigned)p->row_smem;
  k2.kernelParams = a2;
  e = cudaGraphAddKernelNode(&n2, body, &n1, 1, &k2);
  if (e != cudaSuccess) { cudaGraphDestroy(g); cudaGetLastError(); return MGK_CUDA_ERROR; }
  cudaGraphExec_t x = nullptr;
  e = cudaGraphInstantiate(&x, g, 0);
  if (e != cudaSuccess) { cudaGraphDestroy(g); cudaGetLastError(); return MGK_CUDA_ERROR; }
  p->graph = g;
  p->exec = x;
  return MGK_OK;
}

template <typename T>
static int ls2d_solve_t(mgk_ls2d_t p, const double* eb, const double* eps_init, double* eps_out, double* sig_out,
                        int max_iter, double tol, mgk_ls_info* info, cudaStream_t s) {
  const int grid = grid_for(p->N);
  if (eps_init) {
    aos4_partial_kernel<<<grid, 256, 0, s>>>(eps_init, p->N, p->d_part);
    MGK_CUDA(cudaGetLastError());
    finalize_sums_kernel<<<1, 256, 0, s>>>(p->d_part, grid, 4, 1.0 / (double)p->N,
                                           reinterpret_cast<double*>(reinterpret_cast<char*>(p->d_st) +
                                                                     offsetof(Ls2dState, means)));
    MGK_CUDA(cudaGetLastError());
  }
  ls2d_begin_kernel<<<grid, 256, 0, s>>>(p->d_rep, p->d_st, 0, eb[0], eb[1], eb[2], eb[3], eps_init, tol,
                                          max_iter, p->d_part, p->d_counter);
  MGK_CUDA(cudaGetLastError());
  if (eps_init) {
    ls2d_begin_finalize_kernel<<<1, 256, 0, s>>>(p->d_st, 0, p->d_part, grid);
    MGK_CUDA(cudaGetLastError());
  }
  if (max_iter > 0) {
    ls2d_row_kernel<T, false><<<p->row_items, 256, p->row_smem, s>>>(
        p->d_rep, p->d_st, p->d_rowmap, p->d_part, p->d_counter, 1, 0, 0, p->d_any, 0);
    MGK_CUDA(cudaGetLastError());
    if (p->graph_mode == 1 && max_iter + 2 > p->guard_cap) {
      // the loop guard is a graph kernel argument: rebuild for a larger cap
      cudaGraphExecDestroy(p->exec); cudaGraphDestroy(p->graph);
      p->exec = nullptr; p->graph = nullptr; p->graph_mode = -1;
    }
    if (p->graph_mode < 0) {
      const char* env = getenv("MGK_NO_GRAPH_WHILE");
      p->guard_cap = max_iter + 2 > 1000 ? max_iter + 2 : 1000;
      p->graph_mode = (env && env[0] == '1') ? 0 : (ls2d_build_graph<T>(p) == MGK_OK ? 1 : 0);
    }
    if (p->graph_mode == 1) {
      MGK_CUDA(cudaGraphLaunch(p->exec, s));
    } else {
      // host-driven loop: poll the device flag after each iteration
      int* h_any = p->h_any;
      for (int it = 0; it < max_iter; ++it) {
        int st = ls2d_launch_body<T>(p, s, 0, 0);
        if (st) return st;
        MGK_CUDA(cudaMemcpyAsync(h_any, p->d_any, sizeof(int), cudaMemcpyDeviceToHost, s));
        MGK_CUDA(cudaStreamSynchronize(s));
        if (!*h_any) break;
      }
    }
  }
  ls2d_output_kernel<<<grid, 256, 0, s>>>(p->d_rep, p->d_st, 0, eps_out, sig_out, p->d_part);
  MGK_CUDA(cudaGetLastError());
  finalize_sums_kernel<<<1, 256, 0, s>>>(p->d_part, grid, 8, 1.0 / (double)p->N,
                                         reinterpret_cast<double*>(reinterpret_cast<char*>(p->d_st) +
                                                                   offsetof(Ls2dState, out_eps_mean)));
  MGK_CUDA(cudaGetLastError());
  if (info) {
    MGK_CUDA(cudaMemcpyAsync(p->h_state, p->d_st, sizeof(Ls2dState), cudaMemcpyDeviceToHost, s));
    MGK_CUDA(cudaStreamSynchronize(s));
    const Ls2dState& S = *p->h_state;
    info->iterations = S.iter;
    info->status = S.status;
    info->final_diff = S.diff;
    for (int q = 0; q < 4; ++q) { info->eps_mean[q] = S.out_eps_mean[q]; info->sig_mean[q] = S.out_sig_mean[q]; }
    if (S.status == MGK_NONFINITE) {
      set_error("mgk_ls2d_solve: non-finite residual at iteration %d", S.iter);
      return MGK_NONFINITE;
    }
  }
  return MGK_OK;
}

extern "C" int mgk_ls2d_solve(mgk_ls2d_t p, const double* eps_bar, const double* eps_init, double* eps_out,
                              double* sig_out, int max_iter, double tol, mgk_ls_info* info,
                              mgk_stream_t stream) {
  MGK_REQUIRE(p && eps_bar, "mgk_ls2d_solve: null argument");
  MGK_REQUIRE(p->has_material, "mgk_ls2d_solve: call mgk_ls2d_set_material first");
  MGK_REQUIRE(max_iter >= 0 && max_iter <= 1000000, "mgk_ls2d_solve: max_iter out of range");
  cudaStream_t s = (cudaStream_t)stream;
  return p->prec == MGK_FP64 ? ls2d_solve_t<double>(p, eps_bar, eps_init, eps_out, sig_out, max_iter, tol, info, s)
                             : ls2d_solve_t<float>(p, eps_bar, eps_init, eps_out, sig_out, max_iter, tol, info, s);
}

template <typename T>
static int ls2d_profile_t(mgk_ls2d_t p, const double* eb, int reps, float* row_ms, float* col_ms, cudaStream_t s) {
  const int grid = grid_for(p->N);
  ls2d_begin_kernel<<<grid, 256, 0, s>>>(p->d_rep, p->d_st, 0, eb[0], eb[1], eb[2], eb[3], nullptr, 0.0,
                                          1 << 30, p->d_part, p->d_counter);
  MGK_CUDA(cudaGetLastError());
  ls2d_row_kernel<T, false><<<p->row_items, 256, p->row_smem, s>>>(
      p->d_rep, p->d_st, p->d_rowmap, p->d_part, p->d_counter, 1, 0, 0, p->d_any, 0);
  MGK_CUDA(cudaGetLastError());
  cudaEvent_t ev[3];
  for (int i = 0; i < 3; ++i) MGK_CUDA(cudaEventCreate(&ev[i]));
  float tr = 0, tc = 0;
  int rc = MGK_OK;
  for (int r = 0; r < reps && rc == MGK_OK; ++r) {
    cudaEventRecord(ev[0], s);
    ls2d_col_kernel<T><<<p->col_items, 256, p->col_smem, s>>>(p->d_rep, p->d_st, p->d_colmap);
    cudaEventRecord(ev[1], s);
    ls2d_row_kernel<T, true><<<p->row_items, 256, p->row_smem, s>>>(
        p->d_rep, p->d_st, p->d_rowmap, p->d_part, p->d_counter, 1, 0, 0, p->d_any, 0);
    cudaEventRecord(ev[2], s);
    if (cudaEventSynchronize(ev[2]) != cudaSuccess) { rc = MGK_CUDA_ERROR; break; }
    float a = 0, b = 0;
    cudaEventElapsedTime(&a, ev[0], ev[1]);
    cudaEventElapsedTime(&b, ev[1], ev[2]);
    tc += a;
    tr += b;
  }
  for (int i = 0; i < 3; ++i) cudaEventDestroy(ev[i]);
  MGK_CUDA(cudaGetLastError());
  if (rc != MGK_OK) { set_error("mgk_ls2d_profile: kernel failure"); return rc; }
  *row_ms = tr / reps;
  *col_ms = tc / reps;
  return MGK_OK;
}

extern "C" int mgk_ls2d_profile(mgk_ls2d_t p, const double* eps_bar, int reps, float* row_ms, float* col_ms,
                                mgk_stream_t stream) {
  MGK_REQUIRE(p && eps_bar && row_ms && col_ms && reps > 0, "mgk_ls2d_profile: bad argument");
  MGK_REQUIRE(p->has_material, "mgk_ls2d_profile: call mgk_ls2d_set_material first");
  cudaStream_t s = (cudaStream_t)stream;
  return p->prec == MGK_FP64 ? ls2d_profile_t<double>(p, eps_bar, reps, row_ms, col_ms, s)
                             : ls2d_profile_t<float>(p, eps_bar, reps, row_ms, col_ms, s);
}

// ============================================================ no-alloc ===
// Allocation-free 2D LS solve.  Some callers cannot call cudaMalloc: a host
// application or framework whose caching allocator already reserves the
// device memory, a serving process with a fixed memory budget that must not
// allocate after start-up, or code that must avoid the device-wide
// synchronisation cudaFree performs.  For them every buffer the solve needs
// beyond its inputs and outputs lives in one file-scope device array, sized
// for grids up to MGK_NOALLOC_MAX_SIDE per side; each GPU that loads this
// library holds it (about 7 MB) until the process exits.
namespace {
constexpr long long kNaMaxN = (long long)MGK_NOALLOC_MAX_SIDE * MGK_NOALLOC_MAX_SIDE;
constexpr size_t kNaPlanes = 10 * (size_t)kNaMaxN;                                          // 10 real planes
constexpr size_t kNaSpec = 3 * (size_t)MGK_NOALLOC_MAX_SIDE * (MGK_NOALLOC_MAX_SIDE / 2 + 1) * 2;  // complex
constexpr size_t kNaTw = 2 * (size_t)MGK_NOALLOC_MAX_SIDE * 2;                               // two tables
constexpr size_t kNaPart = 8 * 2048;                                                         // partial sums
constexpr size_t kNaMisc = 1024;                    // plan record, state, work maps, counters
constexpr size_t kNaDoubles = kNaPlanes + kNaSpec + kNaTw + kNaPart + kNaMisc;
}  // namespace

// Device-side storage.  In host code this name is only a stand-in for the
// device address, which cudaGetSymbolAddress resolves per device.
static __device__ __align__(256) double g_ls2d_noalloc_scratch[kNaDoubles];

namespace mgk {

// Writes the plan record, clears the work maps, counters and state, and fills
// the twiddle tables (sincospi) -- everything a call must start from.
__global__ void ls2d_noalloc_setup_kernel(Ls2dRep rep, Ls2dRep* dst, Ls2dState* st, int* rowmap, int rowitems,
                                          int* colmap, int colitems, unsigned int* counter, int* any,
                                          double2* twx, int nx, double2* twy, int ny) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int stride = gridDim.x * blockDim.x;
  for (int i = t; i < rowitems; i += stride) rowmap[i] = 0;
  for (int i = t; i < colitems; i += stride) colmap[i] = 0;
  for (int m = t; m < nx; m += stride) {
    double s, c;
    sincospi(2.0 * m / nx, &s, &c);
    twx[m] = make_double2(c, -s);
  }
  for (int m = t; m < ny; m += stride) {
    double s, c;
    sincospi(2.0 * m / ny, &s, &c);
    twy[m] = make_double2(c, -s);
  }
  if (t == 0) {
    *dst = rep;
    counter[0] = 0;
    counter[1] = 0;
    *any = 0;
    Ls2dState z;
    memset(&z, 0, sizeof(z));
    *st = z;
  }
}

}  // namespace mgk

#include <mutex>

static std::mutex g_noalloc_mu;
static void* g_noalloc_addr[128];  // resolved scratch address per device

// First call on a device: resolve the device address of the scratch array
// (this loads the module if it is not loaded yet).  Later calls reuse it.
static int noalloc_scratch(double** out) {
  int dev = -1;
  MGK_CUDA(cudaGetDevice(&dev));
  MGK_REQUIRE(dev >= 0 && dev < 128, "mgk_ls2d_solve_noalloc: device index %d out of range", dev);
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_addr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_ls2d_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr) {
      set_error("mgk_ls2d_solve_noalloc: cudaGetSymbolAddress failed on device %d: %s", dev, cudaGetErrorString(e));
      return MGK_CUDA_ERROR;
    }
    g_noalloc_addr[dev] = p;
  }
  *out = reinterpret_cast<double*>(g_noalloc_addr[dev]);
  return MGK_OK;
}

extern "C" int mgk_ls2d_solve_noalloc(int nx, int ny, int plane_mode, const double* E, const double* nu,
                                      const double* eps_plastic, const double* eps_bar, const double* eps_init,
                                      double* eps_out, double* sig_out, int max_iter, double tol,
                                      mgk_ls_info* info, mgk_stream_t stream) {
  MGK_REQUIRE(nx >= 4 && ny >= 4 && nx <= MGK_NOALLOC_MAX_SIDE && ny <= MGK_NOALLOC_MAX_SIDE,
              "mgk_ls2d_solve_noalloc: grid %dx%d exceeds the maximum of %dx%d for the allocation-free entry "
              "point (use mgk_ls2d_create/mgk_ls2d_solve)", nx, ny, MGK_NOALLOC_MAX_SIDE, MGK_NOALLOC_MAX_SIDE);
  FftLen fx, fy;
  MGK_REQUIRE(fft_schedule(nx, &fx) && fft_schedule(ny, &fy),
              "mgk_ls2d_solve_noalloc: grid %dx%d unsupported (each side must be 2^a 3^b, even)", nx, ny);
  MGK_REQUIRE(plane_mode == MGK_PLANE_STRAIN || plane_mode == MGK_PLANE_STRESS,
              "mgk_ls2d_solve_noalloc: plane_mode must be 0 (strain) or 1 (stress)");
  MGK_REQUIRE(E && nu && eps_bar && eps_out && sig_out, "mgk_ls2d_solve_noalloc: null argument");
  MGK_REQUIRE(max_iter >= 0 && max_iter <= 1000000, "mgk_ls2d_solve_noalloc: max_iter out of range");
  double* base = nullptr;
  int st = noalloc_scratch(&base);
  if (st != MGK_OK) return st;
  cudaStream_t s = (cudaStream_t)stream;

  const long long N = (long long)nx * ny;
  const int nyh = ny / 2 + 1;
  int tc = 8;
  while (tc > 1 && 2 * 3 * (size_t)tc * nx * sizeof(double2) > 200 * 1024) tc >>= 1;
  const int row_items = nx / 2, col_items = (nyh + tc - 1) / tc;
  const size_t row_smem = 2 * 3 * (size_t)ny * sizeof(double2);
  const size_t col_smem = 2 * 3 * (size_t)tc * nx * sizeof(double2);
  MGK_CUDA(cudaFuncSetAttribute(ls2d_row_kernel<double, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)row_smem));
  MGK_CUDA(cudaFuncSetAttribute(ls2d_row_kernel<double, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)row_smem));
  MGK_CUDA(cudaFuncSetAttribute(ls2d_col_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)col_smem));

  // carve the scratch array (offsets in doubles, each region 256-byte aligned)
  double* planes = base;
  double2* spec = reinterpret_cast<double2*>(base + kNaPlanes);
  double2* twx = reinterpret_cast<double2*>(base + kNaPlanes + kNaSpec);
  double2* twy = twx + MGK_NOALLOC_MAX_SIDE;
  double* part = base + kNaPlanes + kNaSpec + kNaTw;
  char* misc = reinterpret_cast<char*>(base + kNaPlanes + kNaSpec + kNaTw + kNaPart);
  Ls2dRep* d_rep = reinterpret_cast<Ls2dRep*>(misc);
  Ls2dState* d_st = reinterpret_cast<Ls2dState*>(misc + 1024);
  int* d_rowmap = reinterpret_cast<int*>(misc + 2048);
  int* d_colmap = reinterpret_cast<int*>(misc + 2048 + 4 * 256);
  unsigned int* d_counter = reinterpret_cast<unsigned int*>(misc + 2048 + 8 * 256);
  int* d_any = reinterpret_cast<int*>(misc + 2048 + 8 * 256 + 64);
  static_assert(sizeof(Ls2dRep) <= 1024 && sizeof(Ls2dState) <= 1024, "no-alloc record sizes");
  static_assert(2048 + 8 * 256 + 128 <= kNaMisc * sizeof(double), "no-alloc misc region");

  fx.tw = twx;
  fy.tw = twy;
  Ls2dRep R;
  memset(&R, 0, sizeof(R));
  R.nx = nx; R.ny = ny; R.nyh = nyh; R.ld = nyh;
  R.row_base = 0; R.row_items = row_items; R.col_base = 0; R.col_items = col_items; R.tc = tc;
  R.N = N; R.fx = fx; R.fy = fy;
  R.mu = planes; R.lam = planes + N; R.eps = planes + 2 * N; R.ep = planes + 5 * N;
  R.epa = eps_plastic ? planes + 8 * N : nullptr;
  R.has_epa = eps_plastic ? 1 : 0;
  R.spec = spec;

  ls2d_noalloc_setup_kernel<<<4, 256, 0, s>>>(R, d_rep, d_st, d_rowmap, row_items, d_colmap, col_items, d_counter,
                                              d_any, twx, nx, twy, ny);
  MGK_CUDA(cudaGetLastError());
  const int grid = grid_for(N);
  ls2d_material_kernel<<<grid, 256, 0, s>>>(d_rep, 0, E, nu, eps_plastic, plane_mode, 1, part);
  MGK_CUDA(cudaGetLastError());
  ls2d_medium_kernel<<<1, 256, 0, s>>>(d_rep, d_st, 0, part, grid, plane_mode);
  MGK_CUDA(cudaGetLastError());
  const double* eb = eps_bar;
  if (eps_init) {
    aos4_partial_kernel<<<grid, 256, 0, s>>>(eps_init, N, part);
    MGK_CUDA(cudaGetLastError());
    finalize_sums_kernel<<<1, 256, 0, s>>>(part, grid, 4, 1.0 / (double)N,
                                           reinterpret_cast<double*>(reinterpret_cast<char*>(d_st) +
                                                                     offsetof(Ls2dState, means)));
    MGK_CUDA(cudaGetLastError());
  }
  ls2d_begin_kernel<<<grid, 256, 0, s>>>(d_rep, d_st, 0, eb[0], eb[1], eb[2], eb[3], eps_init, tol, max_iter, part,
                                          d_counter);
  MGK_CUDA(cudaGetLastError());
  if (eps_init) {
    ls2d_begin_finalize_kernel<<<1, 256, 0, s>>>(d_st, 0, part, grid);
    MGK_CUDA(cudaGetLastError());
  }
  if (max_iter > 0) {
    ls2d_row_kernel<double, false><<<row_items, 256, row_smem, s>>>(d_rep, d_st, d_rowmap, part, d_counter, 1, 0,
                                                                    0, d_any, 0);
    MGK_CUDA(cudaGetLastError());
    // host-driven loop in chunks of 4 iterations; finished iterations skip
    // their work on the device, and the host polls the activity flag
    int it = 0;
    while (it < max_iter) {
      const int chunk = max_iter - it < 4 ? max_iter - it : 4;
      for (int c = 0; c < chunk; ++c) {
        ls2d_col_kernel<double><<<col_items, 256, col_smem, s>>>(d_rep, d_st, d_colmap);
        ls2d_row_kernel<double, true><<<row_items, 256, row_smem, s>>>(d_rep, d_st, d_rowmap, part, d_counter, 1,
                                                                       0, 0, d_any, 0);
      }
      MGK_CUDA(cudaGetLastError());
      it += chunk;
      int h_any = 0;
      MGK_CUDA(cudaMemcpyAsync(&h_any, d_any, sizeof(int), cudaMemcpyDeviceToHost, s));
      MGK_CUDA(cudaStreamSynchronize(s));
      if (!h_any) break;
    }
  }
  ls2d_output_kernel<<<grid, 256, 0, s>>>(d_rep, d_st, 0, eps_out, sig_out, part);
  MGK_CUDA(cudaGetLastError());
  finalize_sums_kernel<<<1, 256, 0, s>>>(part, grid, 8, 1.0 / (double)N,
                                         reinterpret_cast<double*>(reinterpret_cast<char*>(d_st) +
                                                                   offsetof(Ls2dState, out_eps_mean)));
  MGK_CUDA(cudaGetLastError());
  Ls2dState h;
  MGK_CUDA(cudaMemcpyAsync(&h, d_st, sizeof(Ls2dState), cudaMemcpyDeviceToHost, s));
  MGK_CUDA(cudaStreamSynchronize(s));
  if (info) {
    info->iterations = h.iter;
    info->status = h.status;
    info->final_diff = h.diff;
    for (int q = 0; q < 4; ++q) { info->eps_mean[q] = h.out_eps_mean[q]; info->sig_mean[q] = h.out_sig_mean[q]; }
  }
  if (h.status == MGK_NONFINITE) {
    set_error("mgk_ls2d_solve_noalloc: non-finite residual at iteration %d", h.iter);
    return MGK_NONFINITE;
  }
  return MGK_OK;
}
