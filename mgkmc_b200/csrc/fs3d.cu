// 3D finite-strain de Geus Newton-Krylov solver (FP64), matrix-free.
//
// Restates finite_strain_solver_step_3d (mgkmc/finite_strain_simulator.py:
// 2967-3168) with solver="newton_cg": the macro mixed-BC loop, the Newton
// loop with the alpha-halving line search, and the Krylov solve of
//     G : K(F) : dF = rhs,   rhs = -G:K:DbarF (first iteration) or -G:P,
// where G is the de Geus projection (build_ghat4_3d :1121-1167, applied as
// (G:A)_ij = (A^ xi)_i xi_j / |xi|^2, zero at DC and on Nyquist planes) and
// K(F) is applied per voxel from F, F_p^-1 and the moduli without forming
// the 81-component tangent:
//   with F_p:    K:dF = S_ref dF^T + Fp^-1 Y Fe^T,  Y = C_eff : sym(Fe^T dF Fp^-1)
//   without F_p: K:dF = dF S + Fe Y',               Y' = C_eff : sym(Fe^T dF)
// (the two branches of the reference's tangent, :1849-1871).  Materials:
// SVK (the reference's 3D law) and Neo-Hookean (the reference's plane-strain
// law restated in 3D: S = mu I + (lam ln Je - mu) C^-1).  The Krylov solver
// is CG (the operator is symmetric on the range of G); every inner product
// and norm is FP64.
//
// Layout: tensor-first planes like the reference API, F[i][j] is plane
// 3*i+j of N = nx*ny*nz doubles (C order, z fastest).
//
// One matvec = five kernels: zfwd (p update + K:p per voxel + R2C along z of
// pairs of z-lines), y pass, x pass fused with G, inverse y pass, zinv (C2R
// along z + the p.q partial sums).  The CG scalars (alpha, beta, r.r) are
// computed on the device; the host reads r.r once per iteration.
#include <math.h>
#include <stddef.h>
#include <stdlib.h>

#include <algorithm>
#include <vector>

#include "common.cuh"
#include "fft.cuh"

namespace mgk {

const void* twiddles(int n, int prec);

struct FsScalars {
  double rr, pq, alpha, beta, bb;
  double xx, FF, minJe, nan, pad;
  double sig[9];
  double meanF[9];
  double tol2, kmax, kcount;  // device-side CG loop: (tol_CG)^2, iteration cap, iterations run
  double pad2;
};

struct FsArgs {
  int nx, ny, nz, nzh, ld, tc;
  long long N;
  int has_fp, model;  // model 0 SVK, 1 Neo-Hookean
  int plane_stress;   // (nx, 1, ny) plan of a 2D plane-stress solve (lam the plane-stress lambda)
  FftLen fx, fy, fz;
  const double* F;
  const double* Fpi;
  const double* mu;
  const double* lam;
  const double* P;
  double* x;
  double* r;
  double* p;
  double* q;
  double* Fout;
  double* Pout;
  double2* spec;
  double* part;
  FsScalars* sc;
  // FP32 copies for the mixed form's Krylov matvecs
  FftLen fx32, fy32, fz32;
  const float* F32;
  const float* Fpi32;
  const float* mu32;
  const float* lam32;
  float* p32;
  float* q32;
  float* r32;
  float* x32;
  // tangent state at the current F (kFsState planes), FP64 and FP32
  double* st64;
  float* st32;
};

// Tangent state planes: Fe (9), S_ref (6: 00 11 22 12 02 01), C^-1 (6, same
// order; Neo-Hookean only), lambda, c (mu - lambda ln Je for Neo-Hookean, mu
// for SVK), F_p flag (1 where F_p^-1 is not the identity).
constexpr int kFsState = 24;

// the planes and FFT tables a matvec of precision T reads
template <typename T> struct FsP;
template <> struct FsP<double> {
  static __device__ __forceinline__ const double* F(const FsArgs& a) { return a.F; }
  static __device__ __forceinline__ const double* Fpi(const FsArgs& a) { return a.Fpi; }
  static __device__ __forceinline__ const double* lam(const FsArgs& a) { return a.lam; }
  static __device__ __forceinline__ const double* mu(const FsArgs& a) { return a.mu; }
  static __device__ __forceinline__ double* p(const FsArgs& a) { return a.p; }
  static __device__ __forceinline__ double* q(const FsArgs& a) { return a.q; }
  static __device__ __forceinline__ double* r(const FsArgs& a) { return a.r; }
  static __device__ __forceinline__ double* x(const FsArgs& a) { return a.x; }
  static __device__ __forceinline__ double* st(const FsArgs& a) { return a.st64; }
  static __device__ __forceinline__ double2* spec(const FsArgs& a) { return a.spec; }
  static __device__ __forceinline__ const FftLen& fx(const FsArgs& a) { return a.fx; }
  static __device__ __forceinline__ const FftLen& fy(const FsArgs& a) { return a.fy; }
  static __device__ __forceinline__ const FftLen& fz(const FsArgs& a) { return a.fz; }
};
template <> struct FsP<float> {
  static __device__ __forceinline__ const float* F(const FsArgs& a) { return a.F32; }
  static __device__ __forceinline__ const float* Fpi(const FsArgs& a) { return a.Fpi32; }
  static __device__ __forceinline__ const float* lam(const FsArgs& a) { return a.lam32; }
  static __device__ __forceinline__ const float* mu(const FsArgs& a) { return a.mu32; }
  static __device__ __forceinline__ float* p(const FsArgs& a) { return a.p32; }
  static __device__ __forceinline__ float* q(const FsArgs& a) { return a.q32; }
  static __device__ __forceinline__ float* r(const FsArgs& a) { return a.r32; }
  static __device__ __forceinline__ float* x(const FsArgs& a) { return a.x32; }
  static __device__ __forceinline__ float* st(const FsArgs& a) { return a.st32; }
  static __device__ __forceinline__ float2* spec(const FsArgs& a) { return reinterpret_cast<float2*>(a.spec); }
  static __device__ __forceinline__ const FftLen& fx(const FsArgs& a) { return a.fx32; }
  static __device__ __forceinline__ const FftLen& fy(const FsArgs& a) { return a.fy32; }
  static __device__ __forceinline__ const FftLen& fz(const FsArgs& a) { return a.fz32; }
};

// ------------------------------------------------------- 3x3 helpers ---
template <typename T> __device__ __forceinline__ void mm(const T* A, const T* B, T* C) {
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) C[3 * i + j] = A[3 * i] * B[j] + A[3 * i + 1] * B[3 + j] + A[3 * i + 2] * B[6 + j];
}
template <typename T> __device__ __forceinline__ void mtm(const T* A, const T* B, T* C) {  // A^T B
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) C[3 * i + j] = A[i] * B[j] + A[3 + i] * B[3 + j] + A[6 + i] * B[6 + j];
}
template <typename T> __device__ __forceinline__ void mmt(const T* A, const T* B, T* C) {  // A B^T
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j)
      C[3 * i + j] = A[3 * i] * B[3 * j] + A[3 * i + 1] * B[3 * j + 1] + A[3 * i + 2] * B[3 * j + 2];
}
template <typename T> __device__ __forceinline__ T det3(const T* A) {
  return A[0] * (A[4] * A[8] - A[5] * A[7]) - A[1] * (A[3] * A[8] - A[5] * A[6]) + A[2] * (A[3] * A[7] - A[4] * A[6]);
}
template <typename T> __device__ __forceinline__ void inv3(const T* A, T* B) {
  const T d = det3(A);
  const T s = T(1) / d;
  B[0] = (A[4] * A[8] - A[5] * A[7]) * s;
  B[1] = -(A[1] * A[8] - A[2] * A[7]) * s;
  B[2] = (A[1] * A[5] - A[2] * A[4]) * s;
  B[3] = -(A[3] * A[8] - A[5] * A[6]) * s;
  B[4] = (A[0] * A[8] - A[2] * A[6]) * s;
  B[5] = -(A[0] * A[5] - A[2] * A[3]) * s;
  B[6] = (A[3] * A[7] - A[4] * A[6]) * s;
  B[7] = -(A[0] * A[7] - A[1] * A[6]) * s;
  B[8] = (A[0] * A[4] - A[1] * A[3]) * s;
}

// Per-voxel material state at F: Fe, S_ref, and what the tangent needs,
// in arithmetic T (FP64, or FP32 for the mixed form's Krylov matvecs).
template <typename T>
struct VoxelLaw {
  T Fe[9], Fpi[9], Sref[9], S[9], Ci[9];
  T lam, mu, c, Je;
  T f33;  // out-of-plane stretch of a plane-stress plan (1 otherwise)
  int model, has_fp;

  __device__ void init(const FsArgs& a, long long i, const T* F, T alpha, const T* dX) {
    model = a.model;
    has_fp = a.has_fp;
    lam = FsP<T>::lam(a)[i];
    mu = FsP<T>::mu(a)[i];
    T Fv[9];
    for (int q = 0; q < 9; ++q) Fv[q] = F[q] + (dX ? alpha * dX[q] : T(0));
    if (has_fp) {
      const T* fp = FsP<T>::Fpi(a);
      for (int q = 0; q < 9; ++q) Fpi[q] = fp[q * a.N + i];
    } else {
      for (int q = 0; q < 9; ++q) Fpi[q] = (q % 4 == 0) ? T(1) : T(0);
    }
    mm(Fv, Fpi, Fe);
    T C[9];
    mtm(Fe, Fe, C);
    Je = det3(Fe);
    f33 = T(1);
    if (model == 0) {
      T Eg[9];
      for (int q = 0; q < 9; ++q) Eg[q] = T(0.5) * (C[q] - ((q % 4 == 0) ? T(1) : T(0)));
      const T tr = Eg[0] + Eg[4] + Eg[8];
      for (int q = 0; q < 9; ++q) S[q] = 2 * mu * Eg[q] + ((q % 4 == 0) ? lam * tr : T(0));
      if (a.plane_stress) {
        // :1042-1049: E33 = -(lam / (2 mu)) tr E of the in-plane strain (x, z)
        const T e33 = -(lam / (T(2) * mu)) * (Eg[0] + Eg[8]);
        f33 = sqrt(fmax(T(1e-12), T(1) + T(2) * e33));
      }
    } else if (a.plane_stress) {
      // plane-stress Neo-Hookean (:631-684): lam is the plane-stress lambda,
      // lam_3d = 2 mu lam / (2 mu - lam); x = F33^2 from the Newton solve of
      // mu x + lam_3d/2 ln x = mu - lam_3d ln Je (Je of the in-plane Fe, at
      // most 10 steps, until the step is below 1e-12); S = mu I - mu x C^-1;
      // the tangent's lam* = 2 lam_3d mu x / (lam_3d + 2 mu x), c = mu x
      const T lam3 = (T(2) * mu * lam) / fmax(T(1e-14), T(2) * mu - lam);
      const T target = mu - lam3 * log(fmax(T(1e-14), Je));
      T x = T(1);
#pragma unroll 1
      for (int it = 0; it < 10; ++it) {
        const T fx = mu * x + T(0.5) * lam3 * log(x) - target;
        const T dx = -fx / (mu + T(0.5) * lam3 / x);
        x = fmax(T(1e-10), x + dx);
        if (fabs(dx) < T(1e-12)) break;
      }
      f33 = sqrt(fmax(T(1e-12), x));
      inv3(C, Ci);
      c = mu * x;
      for (int q = 0; q < 9; ++q) S[q] = -c * Ci[q] + ((q % 4 == 0) ? mu : T(0));
      lam = (T(2) * lam3 * c) / fmax(T(1e-14), lam3 + T(2) * c);
    } else {
      const T lnJ = log(fmax(T(1e-14), Je));
      inv3(C, Ci);
      c = mu - lam * lnJ;
      const T k = lam * lnJ - mu;
      for (int q = 0; q < 9; ++q) S[q] = k * Ci[q] + ((q % 4 == 0) ? mu : T(0));
    }
    T Tm[9];
    mm(Fpi, S, Tm);
    mmt(Tm, Fpi, Sref);
  }

  // P = Fe S Fp^-T
  __device__ void stress(T* P) const {
    T Tm[9];
    mm(Fe, S, Tm);
    mmt(Tm, Fpi, P);
  }

  // the reference's trans2(K4 : trans2(d))
  __device__ void kdf(const T* d, T* out) const {
    T X[9], Tm[9], Y[9];
    mtm(Fe, d, Tm);
    mm(Tm, Fpi, X);
    if (model == 0) {
      const T tr = X[0] + X[4] + X[8];
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) Y[3 * i + j] = mu * (X[3 * i + j] + X[3 * j + i]) + (i == j ? lam * tr : T(0));
    } else {
      T CX[9], Xs[9], U[9];
      mm(Ci, X, CX);
      const T tr = CX[0] + CX[4] + CX[8];
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) Xs[3 * i + j] = X[3 * i + j] + X[3 * j + i];
      mm(Ci, Xs, U);
      mm(U, Ci, Xs);
      for (int q = 0; q < 9; ++q) Y[q] = lam * tr * Ci[q] + c * Xs[q];
    }
    T A[9], B[9];
    mmt(Sref, d, A);  // S_ref d^T
    mm(Fpi, Y, Tm);
    mmt(Tm, Fe, B);   // Fp^-1 Y Fe^T
    if (has_fp) {
      for (int q = 0; q < 9; ++q) out[q] = A[q] + B[q];
    } else {
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) out[3 * i + j] = A[3 * j + i] + B[3 * j + i];
    }
  }
};

// symmetric 3x3 from its 6 stored components (00 11 22 12 02 01)
template <typename T> __device__ __forceinline__ void sym_load(const T* st, long long N, int off, long long i, T* M) {
  const T a00 = st[(off + 0) * N + i], a11 = st[(off + 1) * N + i], a22 = st[(off + 2) * N + i];
  const T a12 = st[(off + 3) * N + i], a02 = st[(off + 4) * N + i], a01 = st[(off + 5) * N + i];
  M[0] = a00; M[1] = a01; M[2] = a02;
  M[3] = a01; M[4] = a11; M[5] = a12;
  M[6] = a02; M[7] = a12; M[8] = a22;
}

// Tangent state of voxel i at F (FP64 law), stored in precision T.
template <typename T>
__global__ void fs_tangent_kernel(FsArgs a, T* __restrict__ st) {
  const long long N = a.N;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
    double F[9];
    for (int q = 0; q < 9; ++q) F[q] = a.F[q * N + i];
    VoxelLaw<double> law;
    law.init(a, i, F, 0.0, nullptr);
    for (int q = 0; q < 9; ++q) st[q * N + i] = (T)law.Fe[q];
    const int sidx[6] = {0, 4, 8, 5, 2, 1};
    for (int k = 0; k < 6; ++k) st[(9 + k) * N + i] = (T)law.Sref[sidx[k]];
    if (law.model == 1)
      for (int k = 0; k < 6; ++k) st[(15 + k) * N + i] = (T)law.Ci[sidx[k]];
    st[21 * N + i] = (T)law.lam;
    st[22 * N + i] = (T)(law.model == 1 ? law.c : law.mu);
    bool ident = true;
    for (int q = 0; q < 9; ++q) ident = ident && law.Fpi[q] == ((q % 4 == 0) ? 1.0 : 0.0);
    st[23 * N + i] = (T)(ident ? 0 : 1);
  }
}

// trans2(K4 : trans2(d)) from the tangent state (the kdf of VoxelLaw with
// Fe, S_ref, C^-1 precomputed; F_p^-1 read only where the flag is set).
template <typename T>
__device__ __forceinline__ void kdf_state(const FsArgs& a, long long i, const T* d, T* out) {
  const long long N = a.N;
  const T* st = FsP<T>::st(a);
  T Fe[9], Sref[9], X[9], Tm[9], Y[9];
  for (int q = 0; q < 9; ++q) Fe[q] = st[q * N + i];
  sym_load(st, N, 9, i, Sref);
  const T lam = st[21 * N + i], c = st[22 * N + i];
  const bool fp = a.has_fp && st[23 * N + i] != T(0);
  T Fpi[9];
  if (fp) {
    const T* fpp = FsP<T>::Fpi(a);
    for (int q = 0; q < 9; ++q) Fpi[q] = fpp[q * N + i];
  }
  mtm(Fe, d, Tm);
  if (fp) mm(Tm, Fpi, X);
  else for (int q = 0; q < 9; ++q) X[q] = Tm[q];
  if (a.model == 0) {
    const T tr = X[0] + X[4] + X[8];
    for (int r = 0; r < 3; ++r)
      for (int s2 = 0; s2 < 3; ++s2) Y[3 * r + s2] = c * (X[3 * r + s2] + X[3 * s2 + r]) + (r == s2 ? lam * tr : T(0));
  } else {
    T Ci[9], CX[9], Xs[9], U[9];
    sym_load(st, N, 15, i, Ci);
    mm(Ci, X, CX);
    const T tr = CX[0] + CX[4] + CX[8];
    for (int r = 0; r < 3; ++r)
      for (int s2 = 0; s2 < 3; ++s2) Xs[3 * r + s2] = X[3 * r + s2] + X[3 * s2 + r];
    mm(Ci, Xs, U);
    mm(U, Ci, Xs);
    for (int q = 0; q < 9; ++q) Y[q] = lam * tr * Ci[q] + c * Xs[q];
  }
  T A[9], B[9];
  mmt(Sref, d, A);  // S_ref d^T
  if (fp) { mm(Fpi, Y, Tm); mmt(Tm, Fe, B); }
  else mmt(Y, Fe, B);
  if (a.has_fp) {
    for (int q = 0; q < 9; ++q) out[q] = A[q] + B[q];
  } else {
    for (int r = 0; r < 3; ++r)
      for (int s2 = 0; s2 < 3; ++s2) out[3 * r + s2] = A[3 * s2 + r] + B[3 * s2 + r];
  }
}

__device__ __forceinline__ int ffq(int k, int n) { return (k < (n + 1) / 2) ? k : k - n; }

// ----------------------------------------------------------- kernels ---

// z-line forward: MODE 0 CG (p = r + beta p, or p = r when beta = 0; A = K:p),
// 1 uniform (A = K:dbar), 2 residual (A = P).  R2C along z of pairs of
// z-lines, 9 components, in precision T (MODEs 1 and 2 are FP64 only).
template <int MODE, typename T>
__global__ void __launch_bounds__(256) fs_zfwd_kernel(FsArgs a, const double* __restrict__ dbar) {
  using C = C_t<T>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int nz = a.nz, nzh = a.nzh, ld = a.ld;
  const long long N = a.N;
  const long long l0 = 2LL * blockIdx.x;
  const long long plane = (long long)a.nx * a.ny * ld;
  C* bufA = reinterpret_cast<C*>(smem_raw);
  C* bufB = bufA + 9 * nz;
  const double beta = MODE == 0 ? a.sc->beta : 0.0;
  T* pp = FsP<T>::p(a);
  const T* rr = FsP<T>::r(a);
  for (int z = threadIdx.x; z < nz; z += blockDim.x) {
    T out[2][9];
    for (int h = 0; h < 2; ++h) {
      const long long i = (l0 + h) * nz + z;
      if (MODE == 2) {
        for (int q = 0; q < 9; ++q) out[h][q] = (T)a.P[q * N + i];
      } else {
        T d[9];
        if (MODE == 0) {
          for (int q = 0; q < 9; ++q) {
            const double rv = (double)rr[q * N + i];
            const T pn = beta == 0.0 ? (T)rv : (T)(rv + beta * (double)pp[q * N + i]);
            pp[q * N + i] = pn;
            d[q] = pn;
          }
        } else {
          for (int q = 0; q < 9; ++q) d[q] = (T)dbar[q];
        }
        kdf_state<T>(a, i, d, out[h]);
      }
    }
    for (int q = 0; q < 9; ++q) bufA[q * nz + z] = mk<C>(out[0][q], out[1][q]);
  }
  __syncthreads();
  C* Z = fft_any<-1>(bufA, bufB, 9, nz, FsP<T>::fz(a));
  C* spec = FsP<T>::spec(a);
  for (int e = threadIdx.x; e < 9 * nzh; e += blockDim.x) {
    const int c = e / nzh, k = e - c * nzh;
    const C z = Z[c * nz + k];
    const C w = Z[c * nz + (k == 0 ? 0 : nz - k)];
    C* ra = spec + c * plane + l0 * ld;
    ra[k] = mk<C>(T(0.5) * (z.x + w.x), T(0.5) * (z.y - w.y));
    ra[ld + k] = mk<C>(T(0.5) * (z.y + w.y), T(-0.5) * (z.x - w.x));
  }
}

// z-line inverse: C2R along z.  MODE 0: q = result, partial p.q (FP64 sums).
// MODE 1 (FP64): r = -result (right-hand side), x = 0, partial r.r.
template <int MODE, typename T>
__global__ void __launch_bounds__(256) fs_zinv_kernel(FsArgs a) {
  using C = C_t<T>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ double red[32];
  const int nz = a.nz, ld = a.ld;
  const long long N = a.N;
  const long long l0 = 2LL * blockIdx.x;
  const long long plane = (long long)a.nx * a.ny * ld;
  C* bufA = reinterpret_cast<C*>(smem_raw);
  C* bufB = bufA + 9 * nz;
  const C* spec = FsP<T>::spec(a);
  for (int e = threadIdx.x; e < 9 * nz; e += blockDim.x) {
    const int c = e / nz, k = e - c * nz;
    const int ks = (2 * k <= nz) ? k : nz - k;
    const C* ra = spec + c * plane + l0 * ld;
    C av = ra[ks], bv = ra[ld + ks];
    C z;
    if (2 * k <= nz) {
      if (k == 0 || 2 * k == nz) { av.y = 0; bv.y = 0; }
      z = mk<C>(av.x - bv.y, av.y + bv.x);
    } else {
      z = mk<C>(av.x + bv.y, bv.x - av.y);
    }
    bufA[e] = z;
  }
  __syncthreads();
  C* R = fft_any<+1>(bufA, bufB, 9, nz, FsP<T>::fz(a));
  T* qq = FsP<T>::q(a);
  const T* pp = FsP<T>::p(a);
  double acc = 0;
  for (int e = threadIdx.x; e < 9 * nz; e += blockDim.x) {
    const int c = e / nz, z = e - c * nz;
    const C v = R[e];
    for (int h = 0; h < 2; ++h) {
      const long long i = (l0 + h) * nz + z;
      const T val = h == 0 ? v.x : v.y;
      if (MODE == 0) {
        qq[c * N + i] = val;
        acc += (double)pp[c * N + i] * (double)val;
      } else {
        a.r[c * N + i] = -(double)val;
        a.x[c * N + i] = 0.0;
        acc += (double)val * (double)val;
      }
    }
  }
  acc = block_sum(acc, red);
  if (threadIdx.x == 0) a.part[blockIdx.x] = acc;
}

// y-axis pass over tiles of tc kz columns (9 components)
template <int SIGN, typename T>
__global__ void __launch_bounds__(256) fs_ypass_kernel(FsArgs a) {
  using C = C_t<T>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int nx = a.nx, ny = a.ny, nzh = a.nzh, ld = a.ld, tc = a.tc;
  const int ntile = (nzh + tc - 1) / tc;
  const int o = blockIdx.x / ntile;  // x
  const int k0 = (blockIdx.x - o * ntile) * tc;
  const int tcw = min(tc, nzh - k0);
  const long long plane = (long long)nx * ny * ld;
  const long long obase = (long long)o * ny * ld;
  C* bufA = reinterpret_cast<C*>(smem_raw);
  C* bufB = bufA + 9 * tc * ny;
  C* spec = FsP<T>::spec(a);
  const int tot = 9 * tcw * ny;
  for (int e = threadIdx.x; e < tot; e += blockDim.x) {
    const int c = e / (tcw * ny), rem = e - c * tcw * ny, j = rem / tcw, t = rem - j * tcw;
    bufA[(c * tc + t) * ny + j] = spec[c * plane + obase + (long long)j * ld + k0 + t];
  }
  __syncthreads();
  C* F = fft_any<SIGN>(bufA, bufB, 9 * tc, ny, FsP<T>::fy(a));
  for (int e = threadIdx.x; e < tot; e += blockDim.x) {
    const int c = e / (tcw * ny), rem = e - c * tcw * ny, j = rem / tcw, t = rem - j * tcw;
    spec[c * plane + obase + (long long)j * ld + k0 + t] = F[(c * tc + t) * ny + j];
  }
}

// x pass: FFT along x, G, IFFT along x (with the 1/N of the transform pair)
template <typename T>
__global__ void __launch_bounds__(256) fs_xg_kernel(FsArgs a) {
  using C = C_t<T>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int nx = a.nx, ny = a.ny, nz = a.nz, nzh = a.nzh, ld = a.ld, tc = a.tc;
  const int ntile = (nzh + tc - 1) / tc;
  const int o = blockIdx.x / ntile;  // y
  const int k0 = (blockIdx.x - o * ntile) * tc;
  const int tcw = min(tc, nzh - k0);
  const long long plane = (long long)nx * ny * ld;
  const long long lstride = (long long)ny * ld;
  const long long obase = (long long)o * ld;
  C* bufA = reinterpret_cast<C*>(smem_raw);
  C* bufB = bufA + 9 * tc * nx;
  C* spec = FsP<T>::spec(a);
  const int tot = 9 * tcw * nx;
  for (int e = threadIdx.x; e < tot; e += blockDim.x) {
    const int c = e / (tcw * nx), rem = e - c * tcw * nx, j = rem / tcw, t = rem - j * tcw;
    bufA[(c * tc + t) * nx + j] = spec[c * plane + obase + j * lstride + k0 + t];
  }
  __syncthreads();
  C* G = fft_any<-1>(bufA, bufB, 9 * tc, nx, FsP<T>::fx(a));
  const T scale = (T)(1.0 / (double)a.N);
  const int ky = o;
  const double uy = (double)ffq(ky, ny) / ny;
  const bool nqy = (ny & 1) == 0 && 2 * ky == ny;
  for (int e = threadIdx.x; e < tcw * nx; e += blockDim.x) {
    const int t = e / nx, kx = e - t * nx;
    const int kz = k0 + t;
    const bool nqx = (nx & 1) == 0 && 2 * kx == nx, nqz = (nz & 1) == 0 && 2 * kz == nz;
    if ((kx == 0 && ky == 0 && kz == 0) || nqx || nqy || nqz) {
      for (int c = 0; c < 9; ++c) G[(c * tc + t) * nx + kx] = mk<C>(T(0), T(0));
      continue;
    }
    const double ux = (double)ffq(kx, nx) / nx, uz = (double)ffq(kz, nz) / nz;
    const double inv = 1.0 / sqrt(ux * ux + uy * uy + uz * uz);
    const T n[3] = {(T)(ux * inv), (T)(uy * inv), (T)(uz * inv)};
    C A[9];
    for (int c = 0; c < 9; ++c) A[c] = G[(c * tc + t) * nx + kx];
    for (int i = 0; i < 3; ++i) {
      T vx = 0, vy = 0;
      for (int l = 0; l < 3; ++l) { vx += A[3 * i + l].x * n[l]; vy += A[3 * i + l].y * n[l]; }
      for (int j = 0; j < 3; ++j) G[((3 * i + j) * tc + t) * nx + kx] = mk<C>(vx * n[j] * scale, vy * n[j] * scale);
    }
  }
  __syncthreads();
  C* H = (G == bufA) ? bufB : bufA;
  C* Rz = fft_any<+1>(G, H, 9 * tc, nx, FsP<T>::fx(a));
  for (int e = threadIdx.x; e < tot; e += blockDim.x) {
    const int c = e / (tcw * nx), rem = e - c * tcw * nx, j = rem / tcw, t = rem - j * tcw;
    spec[c * plane + obase + j * lstride + k0 + t] = Rz[(c * tc + t) * nx + j];
  }
}

// CG update: x += alpha p; r -= alpha q (the Krylov vectors in the matvec
// precision, FP64 arithmetic and sums); partial r.r
template <typename T>
__global__ void __launch_bounds__(256) fs_update_kernel(FsArgs a) {
  __shared__ double red[32];
  const double alpha = a.sc->alpha;
  const long long n9 = 9 * a.N;
  const T* pp = FsP<T>::p(a);
  const T* qq = FsP<T>::q(a);
  T* xx = FsP<T>::x(a);
  T* rr = FsP<T>::r(a);
  double acc = 0;
  long long start = 0;
  if constexpr (sizeof(T) == 4) {
    // FP32 vectors: four elements per access (16-byte aligned planes)
    const bool vec = ((reinterpret_cast<uintptr_t>(pp) | reinterpret_cast<uintptr_t>(qq) |
                       reinterpret_cast<uintptr_t>(xx) | reinterpret_cast<uintptr_t>(rr)) & 15) == 0;
    if (vec) {
      const long long n4 = n9 / 4;
      const float4* p4 = reinterpret_cast<const float4*>(pp);
      const float4* q4 = reinterpret_cast<const float4*>(qq);
      float4* x4 = reinterpret_cast<float4*>(xx);
      float4* r4 = reinterpret_cast<float4*>(rr);
      for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n4;
           i += (long long)gridDim.x * blockDim.x) {
        const float4 pv = p4[i], qv = q4[i];
        float4 xv = x4[i], rv = r4[i];
        xv.x = (float)((double)xv.x + alpha * (double)pv.x);
        xv.y = (float)((double)xv.y + alpha * (double)pv.y);
        xv.z = (float)((double)xv.z + alpha * (double)pv.z);
        xv.w = (float)((double)xv.w + alpha * (double)pv.w);
        rv.x = (float)((double)rv.x - alpha * (double)qv.x);
        rv.y = (float)((double)rv.y - alpha * (double)qv.y);
        rv.z = (float)((double)rv.z - alpha * (double)qv.z);
        rv.w = (float)((double)rv.w - alpha * (double)qv.w);
        x4[i] = xv;
        r4[i] = rv;
        acc += (double)rv.x * rv.x + (double)rv.y * rv.y + (double)rv.z * rv.z + (double)rv.w * rv.w;
      }
      start = 4 * n4;
    }
  }
  for (long long i = start + blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n9;
       i += (long long)gridDim.x * blockDim.x) {
    xx[i] = (T)((double)xx[i] + alpha * (double)pp[i]);
    const T rn = (T)((double)rr[i] - alpha * (double)qq[i]);
    rr[i] = rn;
    acc += (double)rn * (double)rn;
  }
  acc = block_sum(acc, red);
  if (threadIdx.x == 0) a.part[blockIdx.x] = acc;
}

// fixed-order sum of nb partials; MODE 0: pq -> alpha; 1: r.r -> beta, rr,
// one more Krylov iteration counted; 2: right-hand side -> rr = bb, beta = 0,
// iteration count reset.  MODEs 1 and 2 decide, when use_cond, whether the
// device-side Krylov loop runs another iteration: rr > tol^2 bb, finite, and
// below the iteration cap.
template <int MODE>
__global__ void fs_scalar_kernel(FsArgs a, int nb, cudaGraphConditionalHandle cond, int use_cond) {
  __shared__ double red[32];
  double s = 0;
  for (int i = threadIdx.x; i < nb; i += blockDim.x) s += a.part[i];
  s = block_sum(s, red);
  if (threadIdx.x != 0) return;
  FsScalars& S = *a.sc;
  if (MODE == 0) {
    S.pq = s;
    S.alpha = (s != 0.0) ? S.rr / s : 0.0;
  } else if (MODE == 1) {
    S.beta = (S.rr != 0.0) ? s / S.rr : 0.0;
    S.rr = s;
    S.kcount += 1.0;
  } else {
    S.rr = s;
    S.bb = s;
    S.beta = 0.0;
    S.kcount = 0.0;
  }
  if (MODE != 0 && use_cond) {
    const bool go = isfinite(S.rr) && S.rr > S.tol2 * S.bb && S.kcount < S.kmax;
    cudaGraphSetConditional(cond, go ? 1u : 0u);
  }
}

// Constitutive evaluation at F + alpha (x + dbar) (or at F when dx is 0):
// writes Fout, Pout; per-CTA partials: min Je, NaN count, sum F^2, sum x^2,
// and the Cauchy stress sums (cauchy_from_P_3d).  16 values per CTA.
__global__ void fs_constitutive_kernel(FsArgs a, double alpha, const double* __restrict__ dbar, int use_x) {
  __shared__ double red[32];
  const long long N = a.N;
  double mnJ = INFINITY, nan = 0, FF = 0, xx = 0;
  double sg[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
    double F[9], dX[9];
    for (int q = 0; q < 9; ++q) {
      F[q] = a.F[q * N + i];
      const double xv = use_x ? a.x[q * N + i] : 0.0;
      dX[q] = xv + (dbar ? dbar[q] : 0.0);
      xx += xv * xv;
    }
    VoxelLaw<double> law;
    law.init(a, i, F, alpha, dX);
    double Ft[9], P[9];
    for (int q = 0; q < 9; ++q) Ft[q] = F[q] + alpha * dX[q];
    law.stress(P);
    if (!(law.Je == law.Je)) nan += 1;
    mnJ = fmin(mnJ, law.Je);
    double J = det3(Ft);
    if (a.plane_stress) J *= law.f33;
    if (fabs(J) < 1e-14) J = 1e-14;
    double PF[9];
    mmt(P, Ft, PF);
    for (int q = 0; q < 9; ++q) {
      if (!(P[q] == P[q])) nan += 1;
      a.Fout[q * N + i] = Ft[q];
      a.Pout[q * N + i] = P[q];
      FF += Ft[q] * Ft[q];
      sg[q] += PF[q] / J;
    }
  }
  // min via block reduction on -x with max semantics
  double v[13] = {0};
  v[0] = nan; v[1] = FF; v[2] = xx;
  for (int q = 0; q < 9; ++q) v[3 + q] = sg[q];
  for (int q = 0; q < 12; ++q) {
    const double t = block_sum(v[q], red);
    if (threadIdx.x == 0) a.part[(size_t)blockIdx.x * 16 + q] = t;
  }
  // min Je
  __shared__ double mn[32];
  double m = mnJ;
  for (int o = 16; o > 0; o >>= 1) m = fmin(m, __shfl_down_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) mn[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    double r = INFINITY;
    for (int w = 0; w < (int)(blockDim.x + 31) / 32; ++w) r = fmin(r, mn[w]);
    a.part[(size_t)blockIdx.x * 16 + 12] = r;
  }
}

__global__ void fs_constitutive_finalize(FsArgs a, int nb) {
  __shared__ double red[32];
  __shared__ double mn[32];
  FsScalars& S = *a.sc;
  double v[12];
  for (int q = 0; q < 12; ++q) {
    double s = 0;
    for (int i = threadIdx.x; i < nb; i += blockDim.x) s += a.part[(size_t)i * 16 + q];
    v[q] = block_sum(s, red);
  }
  double m = INFINITY;
  for (int i = threadIdx.x; i < nb; i += blockDim.x) m = fmin(m, a.part[(size_t)i * 16 + 12]);
  for (int o = 16; o > 0; o >>= 1) m = fmin(m, __shfl_down_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) mn[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    double r = INFINITY;
    for (int w = 0; w < (int)(blockDim.x + 31) / 32; ++w) r = fmin(r, mn[w]);
    S.nan = v[0];
    S.FF = v[1];
    S.xx = v[2];
    for (int q = 0; q < 9; ++q) S.sig[q] = v[3 + q] / (double)a.N;
    S.minJe = r;
  }
}

// means of the 9 components of F (DbarF = F_bar - mean(F)): per-CTA partials
__global__ void fs_meanF_kernel(FsArgs a) {
  __shared__ double red[32];
  double s[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < a.N; i += (long long)gridDim.x * blockDim.x)
    for (int q = 0; q < 9; ++q) s[q] += a.F[q * a.N + i];
  for (int q = 0; q < 9; ++q) {
    const double t = block_sum(s[q], red);
    if (threadIdx.x == 0) a.part[(size_t)blockIdx.x * 16 + q] = t;
  }
}

__global__ void fs_meanF_finalize(FsArgs a, int nb) {
  __shared__ double red[32];
  for (int q = 0; q < 9; ++q) {
    double s = 0;
    for (int i = threadIdx.x; i < nb; i += blockDim.x) s += a.part[(size_t)i * 16 + q];
    s = block_sum(s, red);
    if (threadIdx.x == 0) a.sc->meanF[q] = s / (double)a.N;
  }
}

// Cauchy stress field (cauchy_from_P_3d; cauchy_from_P with F33 for plane
// stress), tensor-first
__global__ void fs_cauchy_kernel(FsArgs a, double* sig) {
  const long long N = a.N;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
    double Pv[9], Fv[9], PF[9];
    for (int q = 0; q < 9; ++q) { Pv[q] = a.P[q * N + i]; Fv[q] = a.F[q * N + i]; }
    double J = det3(Fv);
    if (a.plane_stress) {
      VoxelLaw<double> law;
      law.init(a, i, Fv, 0.0, nullptr);
      J *= law.f33;
    }
    if (fabs(J) < 1e-14) J = 1e-14;
    mmt(Pv, Fv, PF);
    for (int q = 0; q < 9; ++q) sig[q * N + i] = PF[q] / J;
  }
}

// Krylov direction and tangent product, per voxel: p = r + beta p (p = r
// when beta = 0), A = K:p from the tangent state, A written to the q planes
// (free until the inverse z pass writes q).  Elementwise at full occupancy;
// the z forward pass (MODE 3) then only transforms A.
template <typename T>
__global__ void __launch_bounds__(256) fs_kp_kernel(FsArgs a) {
  const long long N = a.N;
  const double beta = a.sc->beta;
  T* pp = FsP<T>::p(a);
  const T* rr = FsP<T>::r(a);
  T* qq = FsP<T>::q(a);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
    T d[9], out[9];
    for (int q = 0; q < 9; ++q) {
      const double rv = (double)rr[q * N + i];
      const T pn = beta == 0.0 ? (T)rv : (T)(rv + beta * (double)pp[q * N + i]);
      pp[q * N + i] = pn;
      d[q] = pn;
    }
    kdf_state<T>(a, i, d, out);
    for (int q = 0; q < 9; ++q) qq[q * N + i] = out[q];
  }
}

// ------------------------------------------------- warp-line 3D passes ---
// The same five matvec stages for grids whose sides are 64, 96 or 128 (the
// served and benchmark sizes): lines sit in padded shared memory and
// each warp transforms its own lines with warp-local passes.
//   axis kernels: CTA of NC warps per tile of kFsTile kz columns at one x (y
//     pass) or one y (x pass); warp c transforms component c0 + c's lines.  The
//     x pass applies G between the forward and inverse transforms (CTA
//     barrier); G couples the three components of a row of the tensor only.
//     FP64 CTAs hold 3 components (one row; three CTAs per tile: 5 resident
//     CTAs of 3 warps per SM instead of one of 9 at the registers an FP64 line
//     pair needs), FP32 CTAs all 9.
//   z kernels: CTA of 3 warps per pair of z-lines; the per-voxel stage (K:p or
//     P, or q and the p.q sums) uses all threads, warp w transforms the lines
//     of components 3w..3w+2.
constexpr int kFsTile = 4;

__host__ __device__ constexpr bool fs_fast_len(int n) { return n == 64 || n == 96 || n == 128; }
__host__ __device__ constexpr int fs_pl(int n, int csz) {
  return csz == 16 ? n + n / 8 + 1 : ((n + n / 16 + 2) & ~1);
}

template <int SIGN, typename T, int NL, bool XG, int NC>
__device__ __forceinline__ void fs_axis_body(const FsArgs& a, int o, int k0, int c0, long long obase,
                                             long long jstride, unsigned char* smem) {
  using C = C_t<T>;
  constexpr int PL = padded_len<C>(NL);
  constexpr int TC = kFsTile;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nzh = a.nzh;
  const int tcw = min(TC, nzh - k0);
  const long long plane = (long long)a.nx * a.ny * a.ld;
  C* lines = reinterpret_cast<C*>(smem);  // line (c * TC + t), c relative to c0
  C* spec = FsP<T>::spec(a) + c0 * plane;
  constexpr int TOT = NC * NL * TC;
  for (int e = threadIdx.x; e < TOT; e += NC * 32) {
    const int c = e / (NL * TC);
    const int rem = e - c * NL * TC;
    const int j = rem / TC, t = rem - j * TC;
    if (t < tcw)
      cp_async_elem(&lines[(c * TC + t) * PL + pidx<C>(j)], &spec[c * plane + o * obase + j * jstride + k0 + t]);
  }
  cp_async_wait_all();
  __syncthreads();
  const C* tw = reinterpret_cast<const C*>((XG ? FsP<T>::fx(a) : FsP<T>::fy(a)).tw);
  C* l0 = lines + warp * TC * PL;  // warp = component
  warp_fft<NL, XG ? -1 : SIGN, 2>(l0, PL, tw, lane);
  warp_fft<NL, XG ? -1 : SIGN, 2>(l0 + 2 * PL, PL, tw, lane);
  if constexpr (XG) {
    __syncthreads();
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    const T scale = (T)(1.0 / (double)a.N);
    const int ky = o;
    const double uy = (double)ffq(ky, ny) / ny;
    const bool nqy = (ny & 1) == 0 && 2 * ky == ny;
    for (int e = threadIdx.x; e < tcw * NL; e += NC * 32) {
      const int t = e / NL, kx = e - t * NL;
      const int kz = k0 + t;
      const int pk = pidx<C>(kx);
      const bool nqx = (nx & 1) == 0 && 2 * kx == nx, nqz = (nz & 1) == 0 && 2 * kz == nz;
      if ((kx == 0 && ky == 0 && kz == 0) || nqx || nqy || nqz) {
        for (int c = 0; c < NC; ++c) lines[(c * TC + t) * PL + pk] = mk<C>(T(0), T(0));
        continue;
      }
      const double ux = (double)ffq(kx, nx) / nx, uz = (double)ffq(kz, nz) / nz;
      const double inv = 1.0 / sqrt(ux * ux + uy * uy + uz * uz);
      const T n[3] = {(T)(ux * inv), (T)(uy * inv), (T)(uz * inv)};
      // (G:A)_ij = (A_il n_l) n_j couples the three components of a row of A
      // only: the CTA's NC components are NC / 3 whole rows
      C A[NC];
      for (int c = 0; c < NC; ++c) A[c] = lines[(c * TC + t) * PL + pk];
      for (int i = 0; i < NC / 3; ++i) {
        T vx = 0, vy = 0;
        for (int l = 0; l < 3; ++l) { vx += A[3 * i + l].x * n[l]; vy += A[3 * i + l].y * n[l]; }
        for (int j = 0; j < 3; ++j)
          lines[((3 * i + j) * TC + t) * PL + pk] = mk<C>(vx * n[j] * scale, vy * n[j] * scale);
      }
    }
    __syncthreads();
    warp_fft<NL, +1, 2>(l0, PL, tw, lane);
    warp_fft<NL, +1, 2>(l0 + 2 * PL, PL, tw, lane);
  }
  __syncthreads();
  for (int e = threadIdx.x; e < TOT; e += NC * 32) {
    const int c = e / (NL * TC);
    const int rem = e - c * NL * TC;
    const int j = rem / TC, t = rem - j * TC;
    if (t < tcw) spec[c * plane + o * obase + j * jstride + k0 + t] = lines[(c * TC + t) * PL + pidx<C>(j)];
  }
}

// components per CTA of the axis kernels (FP32 keeps 9: measured faster at
// 128^3), and resident-CTA targets for the register allocator
__host__ __device__ constexpr int fs_axis_nc(bool, int tsz) { return tsz == 4 ? 9 : 3; }
__host__ __device__ constexpr int fs_axis_minb(bool xg, int tsz) { return fs_axis_nc(xg, tsz) == 3 ? 5 : (tsz == 8 ? 1 : 3); }

// y pass (XG = false) or x pass with G (XG = true); grid = (nx or ny) * ntile
// * (9 / NC), the component group fastest
template <int SIGN, typename T, bool XG>
__global__ void __launch_bounds__(fs_axis_nc(XG, sizeof(T)) * 32, fs_axis_minb(XG, sizeof(T)))
    fs_axis_fast_kernel(FsArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  constexpr int NC = fs_axis_nc(XG, sizeof(T));
  const int ntile = (a.nzh + kFsTile - 1) / kFsTile;
  const int cg = blockIdx.x % (9 / NC);
  const int item = blockIdx.x / (9 / NC);
  const int o = item / ntile;
  const int k0 = (item - o * ntile) * kFsTile;
  const long long obase = XG ? (long long)a.ld : (long long)a.ny * a.ld;
  const long long jstride = XG ? (long long)a.ny * a.ld : (long long)a.ld;
  const int nl = XG ? a.nx : a.ny;
#define MGK_AX_CASE(n) case n: fs_axis_body<SIGN, T, n, XG, NC>(a, o, k0, cg * NC, obase, jstride, smem_raw); break;
  switch (nl) {
    MGK_AX_CASE(64) MGK_AX_CASE(96) MGK_AX_CASE(128)
    default: break;
  }
#undef MGK_AX_CASE
}

// z forward: per-voxel stage (MODE 0: p = r + beta p and K:p; 1: K:dbar;
// 2: P; 3: A from the q planes, written by fs_kp_kernel), R2C along z of the
// pair of z-lines, 9 components.
template <int MODE, typename T, int NZ>
__device__ __forceinline__ void fs_zfwd_body(const FsArgs& a, const double* __restrict__ dbar, unsigned char* smem) {
  using C = C_t<T>;
  constexpr int PL = padded_len<C>(NZ);
  constexpr int NZH = NZ / 2 + 1;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long long N = a.N;
  const long long l0 = 2LL * blockIdx.x;
  const long long plane = (long long)a.nx * a.ny * a.ld;
  const int ld = a.ld;
  C* lines = reinterpret_cast<C*>(smem);
  const double beta = MODE == 0 ? a.sc->beta : 0.0;
  T* pp = FsP<T>::p(a);
  const T* rr = FsP<T>::r(a);
  for (int z = threadIdx.x; z < NZ; z += 3 * 32) {
    T out[2][9];
    for (int h = 0; h < 2; ++h) {
      const long long i = (l0 + h) * NZ + z;
      if (MODE == 2) {
        for (int q = 0; q < 9; ++q) out[h][q] = (T)a.P[q * N + i];
      } else if (MODE == 3) {
        const T* qq = FsP<T>::q(a);
        for (int q = 0; q < 9; ++q) out[h][q] = qq[q * N + i];
      } else {
        T d[9];
        if (MODE == 0) {
          for (int q = 0; q < 9; ++q) {
            const double rv = (double)rr[q * N + i];
            const T pn = beta == 0.0 ? (T)rv : (T)(rv + beta * (double)pp[q * N + i]);
            pp[q * N + i] = pn;
            d[q] = pn;
          }
        } else {
          for (int q = 0; q < 9; ++q) d[q] = (T)dbar[q];
        }
        kdf_state<T>(a, i, d, out[h]);
      }
    }
    const int pz = pidx<C>(z);
    for (int q = 0; q < 9; ++q) lines[q * PL + pz] = mk<C>(out[0][q], out[1][q]);
  }
  __syncthreads();
  const C* tw = reinterpret_cast<const C*>(FsP<T>::fz(a).tw);
  C* lw = lines + 3 * warp * PL;
  warp_fft<NZ, -1, 3>(lw, PL, tw, lane);
  C* spec = FsP<T>::spec(a);
  for (int cc = 0; cc < 3; ++cc) {
    const int c = 3 * warp + cc;
    const C* ln = lines + c * PL;
    C* ra = spec + c * plane + l0 * ld;
    for (int k = lane; k < NZH; k += 32) {
      const C zz = ln[pidx<C>(k)];
      const C w = ln[pidx<C>(k == 0 ? 0 : NZ - k)];
      ra[k] = mk<C>(T(0.5) * (zz.x + w.x), T(0.5) * (zz.y - w.y));
      ra[ld + k] = mk<C>(T(0.5) * (zz.y + w.y), T(-0.5) * (zz.x - w.x));
    }
  }
}

template <int MODE, typename T>
__global__ void __launch_bounds__(3 * 32) fs_zfwd_fast_kernel(FsArgs a, const double* __restrict__ dbar) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
#define MGK_ZF_CASE(n) case n: fs_zfwd_body<MODE, T, n>(a, dbar, smem_raw); break;
  switch (a.nz) {
    MGK_ZF_CASE(64) MGK_ZF_CASE(96) MGK_ZF_CASE(128)
    default: break;
  }
#undef MGK_ZF_CASE
}

// z inverse: C2R along z of the pair of z-lines; MODE 0: q and the p.q
// partial; MODE 1 (FP64): r = -result, x = 0, the r.r partial.
template <int MODE, typename T, int NZ>
__device__ __forceinline__ void fs_zinv_body(const FsArgs& a, unsigned char* smem, double* red) {
  using C = C_t<T>;
  constexpr int PL = padded_len<C>(NZ);
  constexpr int NZH = NZ / 2 + 1;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long long N = a.N;
  const long long l0 = 2LL * blockIdx.x;
  const long long plane = (long long)a.nx * a.ny * a.ld;
  const int ld = a.ld;
  C* lines = reinterpret_cast<C*>(smem);
  const C* spec = FsP<T>::spec(a);
  constexpr int U = (NZH + 31) / 32;
  for (int cc = 0; cc < 3; ++cc) {
    const int c = 3 * warp + cc;
    C* ln = lines + c * PL;
    const C* ra = spec + c * plane + l0 * ld;
    // the component's half-spectrum rows into registers first: one memory
    // round trip, not one per strided step behind the shared-memory stores
    C av[U], bv[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int k = lane + 32 * u;
      if (k < NZH) { av[u] = ra[k]; bv[u] = ra[ld + k]; }
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int k = lane + 32 * u;
      if (k < NZH) {
        C x = av[u], y = bv[u];
        if (k == 0 || 2 * k == NZ) { x.y = 0; y.y = 0; }
        ln[pidx<C>(k)] = mk<C>(x.x - y.y, x.y + y.x);
        if (k > 0 && 2 * k < NZ) ln[pidx<C>(NZ - k)] = mk<C>(x.x + y.y, y.x - x.y);
      }
    }
  }
  __syncwarp();
  const C* tw = reinterpret_cast<const C*>(FsP<T>::fz(a).tw);
  warp_fft<NZ, +1, 3>(lines + 3 * warp * PL, PL, tw, lane);
  __syncthreads();
  T* qq = FsP<T>::q(a);
  const T* pp = FsP<T>::p(a);
  double acc = 0;
  for (int z = threadIdx.x; z < NZ; z += 3 * 32) {
    const int pz = pidx<C>(z);
    for (int c = 0; c < 9; ++c) {
      const C v = lines[c * PL + pz];
      for (int h = 0; h < 2; ++h) {
        const long long i = (l0 + h) * NZ + z;
        const T val = h == 0 ? v.x : v.y;
        if (MODE == 0) {
          qq[c * N + i] = val;
          acc += (double)pp[c * N + i] * (double)val;
        } else {
          a.r[c * N + i] = -(double)val;
          a.x[c * N + i] = 0.0;
          acc += (double)val * (double)val;
        }
      }
    }
  }
  acc = block_sum(acc, red);
  if (threadIdx.x == 0) a.part[blockIdx.x] = acc;
}

template <int MODE, typename T>
__device__ __forceinline__ void fs_zinv_fast_entry(const FsArgs& a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ double red[32];
#define MGK_ZI_CASE(n) case n: fs_zinv_body<MODE, T, n>(a, smem_raw, red); break;
  switch (a.nz) {
    MGK_ZI_CASE(64) MGK_ZI_CASE(96) MGK_ZI_CASE(128)
    default: break;
  }
#undef MGK_ZI_CASE
}

// FP32 kernel (the compiler's own register target), and the FP64 kernel with
// a register target of 5 resident CTAs per SM (measured faster than 4 at
// 128^3 despite a few spilled registers; the forward z pass is not)
template <int MODE, typename T>
__global__ void __launch_bounds__(3 * 32) fs_zinv_fast_kernel(FsArgs a) { fs_zinv_fast_entry<MODE, T>(a); }
template <int MODE>
__global__ void __launch_bounds__(3 * 32, 5) fs_zinv_fast64_kernel(FsArgs a) { fs_zinv_fast_entry<MODE, double>(a); }
template <int MODE, typename T> static void* fs_zinv_fast_fn() {
  if constexpr (sizeof(T) == 8) return (void*)fs_zinv_fast64_kernel<MODE>;
  else return (void*)fs_zinv_fast_kernel<MODE, T>;
}

// FP64 copies of n floats (the mixed form's Krylov solution back to FP64)
__global__ void fs_to_f64_kernel(long long n, const float* __restrict__ src, double* __restrict__ dst) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    dst[i] = (double)src[i];
}

// FP32 copies of n doubles (the mixed form's matvec inputs)
__global__ void fs_to_f32_kernel(long long n, const double* __restrict__ src, float* __restrict__ dst) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    dst[i] = (float)src[i];
}

// material: lam, mu planes and Fp^-1 (plain inverse of F_p, as _invert_Fp_3d)
__global__ void fs_material_kernel(long long N, const double* __restrict__ lam_in, const double* __restrict__ mu_in,
                                   const double* __restrict__ Fp, double* lam, double* mu, double* Fpi) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
    lam[i] = lam_in[i];
    mu[i] = mu_in[i];
    if (Fp) {
      double A[9], B[9];
      for (int q = 0; q < 9; ++q) A[q] = Fp[q * N + i];
      double d = det3(A);
      if (fabs(d) < 1e-14) d = 1e-14;
      const double s = 1.0 / d;
      B[0] = (A[4] * A[8] - A[5] * A[7]) * s;
      B[1] = -(A[1] * A[8] - A[2] * A[7]) * s;
      B[2] = (A[1] * A[5] - A[2] * A[4]) * s;
      B[3] = -(A[3] * A[8] - A[5] * A[6]) * s;
      B[4] = (A[0] * A[8] - A[2] * A[6]) * s;
      B[5] = -(A[0] * A[5] - A[2] * A[3]) * s;
      B[6] = (A[3] * A[7] - A[4] * A[6]) * s;
      B[7] = -(A[0] * A[7] - A[1] * A[6]) * s;
      B[8] = (A[0] * A[4] - A[1] * A[3]) * s;
      for (int q = 0; q < 9; ++q) Fpi[q * N + i] = B[q];
    }
  }
}

}  // namespace mgk

// ================================================================== plan ===
using namespace mgk;

struct mgk_fs3d_plan {
  int nx, ny, nz, nzh, ld, tc, model;
  long long N;
  int has_fp = 0, has_material = 0;
  FftLen fx, fy, fz;
  double* fields = nullptr;  // F, Ftr, Fpi, lam, mu, P, Ptr, x, r, p, q
  double *F, *Ftr, *Fpi, *lam, *mu, *P, *Ptr, *x, *r, *p, *q;
  double2* spec = nullptr;
  double* part = nullptr;
  double* dbar = nullptr;   // device 9 doubles
  FsScalars* sc = nullptr;
  FsScalars* h_sc = nullptr;  // pinned
  double* h_dbar = nullptr;   // pinned
  size_t zsmem = 0, ysmem = 0, xsmem = 0;
  int nblk = 0;
  int stat_newton = 0, stat_krylov = 0, stat_macro = 0;
  // precision form: MGK_FP64, or MGK_MIXED (FP32 Krylov matvecs)
  int prec = MGK_FP64;
  float* f32 = nullptr;  // F32, Fpi32, lam32, mu32, p32, q32
  float *F32 = nullptr, *Fpi32 = nullptr, *lam32 = nullptr, *mu32 = nullptr, *p32 = nullptr, *q32 = nullptr;
  float *r32 = nullptr, *x32 = nullptr;
  double* st64 = nullptr;  // tangent state planes (kFsState each)
  float* st32 = nullptr;
  FftLen fx32, fy32, fz32;
  // device-side Krylov loop graphs, one per matvec precision (0 FP64, 1 FP32)
  cudaGraph_t cg_graph[2] = {nullptr, nullptr};
  cudaGraphExec_t cg_exec[2] = {nullptr, nullptr};
  int graph_mode = -1;  // -1 untried, 1 graphs, 0 host-driven loop
  int fast = 0;         // warp-line passes (every side has a compiled FFT)
  // plane strain embedded as (nx, 1, ny): the out-of-plane F_yy = 1 adds N
  // to ||F||^2, which the 2D solver's Newton norm does not contain
  double ff_offset = 0.0;
  int plane_stress = 0;  // 2D plane stress on the (nx, 1, ny) plan
};

static FsArgs fs_args(mgk_fs3d_t p) {
  FsArgs a;
  memset(&a, 0, sizeof(a));
  a.nx = p->nx; a.ny = p->ny; a.nz = p->nz; a.nzh = p->nzh; a.ld = p->ld; a.tc = p->tc;
  a.N = p->N; a.has_fp = p->has_fp; a.model = p->model; a.plane_stress = p->plane_stress;
  a.fx = p->fx; a.fy = p->fy; a.fz = p->fz;
  a.F = p->F; a.Fpi = p->Fpi; a.mu = p->mu; a.lam = p->lam; a.P = p->P;
  a.x = p->x; a.r = p->r; a.p = p->p; a.q = p->q; a.Fout = p->Ftr; a.Pout = p->Ptr;
  a.spec = p->spec; a.part = p->part; a.sc = p->sc;
  a.fx32 = p->fx32; a.fy32 = p->fy32; a.fz32 = p->fz32;
  a.F32 = p->F32; a.Fpi32 = p->Fpi32; a.mu32 = p->mu32; a.lam32 = p->lam32; a.p32 = p->p32; a.q32 = p->q32;
  a.r32 = p->r32; a.x32 = p->x32;
  a.st64 = p->st64; a.st32 = p->st32;
  return a;
}

extern "C" int mgk_fs3d_destroy(mgk_fs3d_t p) {
  if (!p) return MGK_OK;
  for (int k = 0; k < 2; ++k) {
    if (p->cg_exec[k]) cudaGraphExecDestroy(p->cg_exec[k]);
    if (p->cg_graph[k]) cudaGraphDestroy(p->cg_graph[k]);
  }
  cudaFree(p->f32);
  cudaFree(p->st64);
  cudaFree(p->st32);
  cudaFree(p->fields);
  cudaFree(p->spec);
  cudaFree(p->part);
  cudaFree(p->dbar);
  cudaFree(p->sc);
  if (p->h_sc) cudaFreeHost(p->h_sc);
  if (p->h_dbar) cudaFreeHost(p->h_dbar);
  delete p;
  return MGK_OK;
}

extern "C" int mgk_fs3d_create(int nx, int ny, int nz, int model, mgk_fs3d_t* out) {
  MGK_REQUIRE(out, "mgk_fs3d_create: null output handle");
  *out = nullptr;
  MGK_REQUIRE(model == 0 || model == 1, "mgk_fs3d_create: model must be 0 (SVK) or 1 (Neo-Hookean)");
  FftLen fx, fy, fz;
  MGK_REQUIRE(fft_schedule(nx, &fx) && fft_schedule(ny, &fy) && fft_schedule(nz, &fz) && ((long long)nx * ny) % 2 == 0,
              "mgk_fs3d_create: grid %dx%dx%d unsupported (sides 2^a 3^b up to 4096, nx*ny even)", nx, ny, nz);
  mgk_fs3d_t p = new mgk_fs3d_plan();
  auto fail = [&](int s) { mgk_fs3d_destroy(p); return s; };
  p->nx = nx; p->ny = ny; p->nz = nz; p->nzh = nz / 2 + 1; p->ld = p->nzh; p->model = model;
  p->N = (long long)nx * ny * nz;
  int tc = 4;
  while (tc > 1 && 2 * 9 * (size_t)tc * std::max(nx, ny) * sizeof(double2) > 96 * 1024) tc >>= 1;
  p->tc = tc;
  p->zsmem = 2 * 9 * (size_t)nz * sizeof(double2);
  p->ysmem = 2 * 9 * (size_t)tc * ny * sizeof(double2);
  p->xsmem = 2 * 9 * (size_t)tc * nx * sizeof(double2);
  MGK_REQUIRE(p->zsmem <= 220 * 1024 && p->ysmem <= 220 * 1024 && p->xsmem <= 220 * 1024,
              "mgk_fs3d_create: grid too large for the shared-memory FFT");
  fx.tw = twiddles(nx, MGK_FP64); fy.tw = twiddles(ny, MGK_FP64); fz.tw = twiddles(nz, MGK_FP64);
  if (!fx.tw || !fy.tw || !fz.tw) return fail(MGK_OOM);
  p->fx = fx; p->fy = fy; p->fz = fz;
  const long long N = p->N;
  if (cudaMalloc(&p->fields, sizeof(double) * N * (9 * 9 + 2)) != cudaSuccess) { cudaGetLastError(); return fail(MGK_OOM); }
  double* f = p->fields;
  p->F = f; p->Ftr = f + 9 * N; p->Fpi = f + 18 * N; p->lam = f + 27 * N; p->mu = f + 28 * N;
  p->P = f + 29 * N; p->Ptr = f + 38 * N; p->x = f + 47 * N; p->r = f + 56 * N; p->p = f + 65 * N; p->q = f + 74 * N;
  if (cudaMalloc(&p->spec, 9 * (size_t)nx * ny * p->ld * sizeof(double2)) != cudaSuccess) { cudaGetLastError(); return fail(MGK_OOM); }
  if (cudaMalloc(&p->st64, sizeof(double) * kFsState * N) != cudaSuccess) { cudaGetLastError(); return fail(MGK_OOM); }
  p->nblk = (int)std::max(1LL, std::min(1024LL, (N + 255) / 256));
  const size_t npart = std::max((size_t)16 * p->nblk, (size_t)((long long)nx * ny / 2 + 16));
  const size_t npart2 = std::max(npart, (size_t)(9 * N / 256 + 64));
  if (cudaMalloc(&p->part, sizeof(double) * npart2) != cudaSuccess ||
      cudaMalloc(&p->dbar, sizeof(double) * 16) != cudaSuccess || cudaMalloc(&p->sc, sizeof(FsScalars)) != cudaSuccess) {
    cudaGetLastError();
    return fail(MGK_OOM);
  }
  if (cudaMallocHost(&p->h_sc, sizeof(FsScalars)) != cudaSuccess || cudaMallocHost(&p->h_dbar, sizeof(double) * 16) != cudaSuccess)
    return fail(MGK_OOM);
  if (cudaMemset(p->fields, 0, sizeof(double) * N * (9 * 9 + 2)) != cudaSuccess ||
      cudaMemset(p->sc, 0, sizeof(FsScalars)) != cudaSuccess)
    return fail(MGK_CUDA_ERROR);
  if (raise_smem((const void*)fs_zfwd_kernel<0, double>, (int)p->zsmem) ||
      raise_smem((const void*)fs_zfwd_kernel<1, double>, (int)p->zsmem) ||
      raise_smem((const void*)fs_zfwd_kernel<2, double>, (int)p->zsmem) ||
      raise_smem((const void*)fs_zinv_kernel<0, double>, (int)p->zsmem) ||
      raise_smem((const void*)fs_zinv_kernel<1, double>, (int)p->zsmem) ||
      raise_smem((const void*)fs_ypass_kernel<-1, double>, (int)p->ysmem) ||
      raise_smem((const void*)fs_ypass_kernel<1, double>, (int)p->ysmem) ||
      raise_smem((const void*)fs_xg_kernel<double>, (int)p->xsmem) ||
      raise_smem((const void*)fs_zfwd_kernel<0, float>, (int)p->zsmem / 2) ||
      raise_smem((const void*)fs_zinv_kernel<0, float>, (int)p->zsmem / 2) ||
      raise_smem((const void*)fs_ypass_kernel<-1, float>, (int)p->ysmem / 2) ||
      raise_smem((const void*)fs_ypass_kernel<1, float>, (int)p->ysmem / 2) ||
      raise_smem((const void*)fs_xg_kernel<float>, (int)p->xsmem / 2)) {
    set_error("mgk_fs3d_create: cudaFuncSetAttribute failed");
    return fail(MGK_CUDA_ERROR);
  }
  {
    const char* env = getenv("MGK_FS_FAST");
    p->fast = fs_fast_len(nx) && fs_fast_len(ny) && fs_fast_len(nz) && !(env && env[0] == '0');
  }
  if (p->fast) {
    const int zs64 = 9 * fs_pl(nz, 16) * 16, zs32 = 9 * fs_pl(nz, 8) * 8;
    const int ys64 = fs_axis_nc(false, 8) * kFsTile * fs_pl(ny, 16) * 16;
    const int ys32 = fs_axis_nc(false, 4) * kFsTile * fs_pl(ny, 8) * 8;
    const int xs64 = fs_axis_nc(true, 8) * kFsTile * fs_pl(nx, 16) * 16;
    const int xs32 = fs_axis_nc(true, 4) * kFsTile * fs_pl(nx, 8) * 8;
    if (raise_smem((const void*)fs_zfwd_fast_kernel<0, double>, zs64) ||
        raise_smem((const void*)fs_zfwd_fast_kernel<1, double>, zs64) ||
        raise_smem((const void*)fs_zfwd_fast_kernel<2, double>, zs64) ||
        raise_smem((const void*)fs_zfwd_fast_kernel<0, float>, zs32) ||
        raise_smem((const void*)fs_zfwd_fast_kernel<3, double>, zs64) ||
        raise_smem((const void*)fs_zfwd_fast_kernel<3, float>, zs32) ||
        raise_smem(fs_zinv_fast_fn<0, double>(), zs64) ||
        raise_smem(fs_zinv_fast_fn<1, double>(), zs64) ||
        raise_smem((const void*)fs_zinv_fast_kernel<0, float>, zs32) ||
        raise_smem((const void*)fs_axis_fast_kernel<-1, double, false>, ys64) ||
        raise_smem((const void*)fs_axis_fast_kernel<1, double, false>, ys64) ||
        raise_smem((const void*)fs_axis_fast_kernel<-1, double, true>, xs64) ||
        raise_smem((const void*)fs_axis_fast_kernel<-1, float, false>, ys32) ||
        raise_smem((const void*)fs_axis_fast_kernel<1, float, false>, ys32) ||
        raise_smem((const void*)fs_axis_fast_kernel<-1, float, true>, xs32)) {
      set_error("mgk_fs3d_create: cudaFuncSetAttribute failed");
      return fail(MGK_CUDA_ERROR);
    }
  }
  *out = p;
  return MGK_OK;
}

static void fs_drop_graphs(mgk_fs3d_t p) {
  for (int k = 0; k < 2; ++k) {
    if (p->cg_exec[k]) cudaGraphExecDestroy(p->cg_exec[k]);
    if (p->cg_graph[k]) cudaGraphDestroy(p->cg_graph[k]);
    p->cg_exec[k] = nullptr;
    p->cg_graph[k] = nullptr;
  }
}

// FP32 copy of F_p^-1 for the mixed form's matvecs (read where the tangent
// state flags a non-identity F_p)
static int fs_refresh_f32(mgk_fs3d_t p, bool material, cudaStream_t s) {
  if (p->prec != MGK_MIXED || !material || !p->has_fp) return MGK_OK;
  fs_to_f32_kernel<<<p->nblk, 256, 0, s>>>(9 * p->N, p->Fpi, p->Fpi32);
  MGK_CUDA(cudaGetLastError());
  return MGK_OK;
}

// tangent state at the current F (once per accepted Newton iterate; every
// Krylov matvec of the next Newton step reads it)
static int fs_tangent(mgk_fs3d_t p, cudaStream_t s) {
  FsArgs a = fs_args(p);
  fs_tangent_kernel<double><<<p->nblk, 256, 0, s>>>(a, p->st64);
  if (p->prec == MGK_MIXED) fs_tangent_kernel<float><<<p->nblk, 256, 0, s>>>(a, p->st32);
  MGK_CUDA(cudaGetLastError());
  return MGK_OK;
}

extern "C" int mgk_fs3d_set_precision(mgk_fs3d_t p, int precision) {
  MGK_REQUIRE(p, "mgk_fs3d_set_precision: null plan");
  MGK_REQUIRE(precision == MGK_FP64 || precision == MGK_MIXED, "mgk_fs3d_set_precision: bad precision");
  if (precision == MGK_MIXED && !p->f32) {
    const long long N = p->N;
    if (cudaMalloc(&p->f32, sizeof(float) * N * (9 + 9 + 2 + 9 + 9 + 9 + 9)) != cudaSuccess) {
      cudaGetLastError();
      set_error("mgk_fs3d_set_precision: cudaMalloc of the FP32 planes failed");
      return MGK_OOM;
    }
    float* f = p->f32;
    p->F32 = f; p->Fpi32 = f + 9 * N; p->lam32 = f + 18 * N; p->mu32 = f + 19 * N; p->p32 = f + 20 * N;
    p->q32 = f + 29 * N; p->r32 = f + 38 * N; p->x32 = f + 47 * N;
    if (cudaMalloc(&p->st32, sizeof(float) * kFsState * N) != cudaSuccess) {
      cudaGetLastError();
      set_error("mgk_fs3d_set_precision: cudaMalloc of the FP32 tangent state failed");
      return MGK_OOM;
    }
    p->fx32 = p->fx; p->fy32 = p->fy; p->fz32 = p->fz;
    p->fx32.tw = twiddles(p->nx, 1); p->fy32.tw = twiddles(p->ny, 1); p->fz32.tw = twiddles(p->nz, 1);
    if (!p->fx32.tw || !p->fy32.tw || !p->fz32.tw) return MGK_OOM;
  }
  if (precision != p->prec) fs_drop_graphs(p);  // the graphs capture the plane set
  p->prec = precision;
  if (precision == MGK_MIXED && p->has_material) {
    MGK_CUDA(cudaDeviceSynchronize());
    int rc = fs_refresh_f32(p, true, 0);
    if (rc) return rc;
    MGK_CUDA(cudaDeviceSynchronize());
  }
  return MGK_OK;
}

extern "C" int mgk_fs3d_set_material(mgk_fs3d_t p, const double* lam, const double* mu, const double* Fp,
                                     mgk_stream_t stream) {
  MGK_REQUIRE(p && lam && mu, "mgk_fs3d_set_material: null argument");
  cudaStream_t s = (cudaStream_t)stream;
  fs_material_kernel<<<p->nblk, 256, 0, s>>>(p->N, lam, mu, Fp, p->lam, p->mu, p->Fpi);
  MGK_CUDA(cudaGetLastError());
  if ((Fp ? 1 : 0) != p->has_fp) fs_drop_graphs(p);  // the graphs capture has_fp
  p->has_fp = Fp ? 1 : 0;
  p->has_material = 1;
  return fs_refresh_f32(p, true, s);
}

extern "C" int mgk_fs3d_set_F(mgk_fs3d_t p, const double* F, mgk_stream_t stream) {
  MGK_REQUIRE(p && F, "mgk_fs3d_set_F: null argument");
  MGK_CUDA(cudaMemcpyAsync(p->F, F, sizeof(double) * 9 * p->N, cudaMemcpyDeviceToDevice, (cudaStream_t)stream));
  return MGK_OK;
}

extern "C" int mgk_fs3d_get(mgk_fs3d_t p, double* F_out, double* P_out, double* sig_out, mgk_stream_t stream) {
  MGK_REQUIRE(p, "mgk_fs3d_get: null plan");
  cudaStream_t s = (cudaStream_t)stream;
  if (F_out) MGK_CUDA(cudaMemcpyAsync(F_out, p->F, sizeof(double) * 9 * p->N, cudaMemcpyDeviceToDevice, s));
  if (P_out) MGK_CUDA(cudaMemcpyAsync(P_out, p->P, sizeof(double) * 9 * p->N, cudaMemcpyDeviceToDevice, s));
  if (sig_out) {
    fs_cauchy_kernel<<<p->nblk, 256, 0, s>>>(fs_args(p), sig_out);
    MGK_CUDA(cudaGetLastError());
  }
  return MGK_OK;
}

// The five launches of one matvec / projection (function, grid, block,
// shared memory), for the plan's kernel family and precision T.
struct FsLaunch {
  void* fn;
  dim3 grid, block;
  size_t smem;
  int args;  // 0: (FsArgs), 1: (FsArgs, dbar)
};
// returns the number of launches (5, or 6 when the tangent product runs as
// its own elementwise kernel)
template <typename T>
static int fs_stage_launches(mgk_fs3d_t p, int mode, int zmode, FsLaunch L[6]) {
  const int zl = (int)(p->N / p->nz / 2);
  int k = 0;
  if (p->fast) {
    const int csz = (int)sizeof(C_t<T>);
    const int ntile = (p->nzh + kFsTile - 1) / kFsTile;
    const size_t zs = 9 * (size_t)fs_pl(p->nz, csz) * csz, zs64 = 9 * (size_t)fs_pl(p->nz, 16) * 16;
    constexpr int ncy = fs_axis_nc(false, sizeof(T)), ncx = fs_axis_nc(true, sizeof(T));
    const size_t ys = ncy * (size_t)kFsTile * fs_pl(p->ny, csz) * csz;
    const size_t xs = ncx * (size_t)kFsTile * fs_pl(p->nx, csz) * csz;
    if (mode == 0) {
      L[k++] = {(void*)fs_kp_kernel<T>, dim3(4 * p->nblk), dim3(256), 0, 0};
      L[k++] = {(void*)fs_zfwd_fast_kernel<3, T>, dim3(zl), dim3(96), zs, 1};
    } else {
      L[k++] = {mode == 1 ? (void*)fs_zfwd_fast_kernel<1, double> : (void*)fs_zfwd_fast_kernel<2, double>, dim3(zl),
                dim3(96), zs64, 1};
    }
    L[k++] = {(void*)fs_axis_fast_kernel<-1, T, false>, dim3(p->nx * ntile * (9 / ncy)), dim3(32 * ncy), ys, 0};
    L[k++] = {(void*)fs_axis_fast_kernel<-1, T, true>, dim3(p->ny * ntile * (9 / ncx)), dim3(32 * ncx), xs, 0};
    L[k++] = {(void*)fs_axis_fast_kernel<1, T, false>, dim3(p->nx * ntile * (9 / ncy)), dim3(32 * ncy), ys, 0};
    L[k++] = {zmode == 0 ? fs_zinv_fast_fn<0, T>() : fs_zinv_fast_fn<1, double>(), dim3(zl),
              dim3(96), zmode == 0 ? zs : zs64, 0};
  } else {
    const int ntile = (p->nzh + p->tc - 1) / p->tc;
    const size_t zs = p->zsmem * sizeof(T) / 8, ys = p->ysmem * sizeof(T) / 8, xs = p->xsmem * sizeof(T) / 8;
    L[k++] = {mode == 0 ? (void*)fs_zfwd_kernel<0, T>
                        : (mode == 1 ? (void*)fs_zfwd_kernel<1, double> : (void*)fs_zfwd_kernel<2, double>),
              dim3(zl), dim3(256), mode == 0 ? zs : p->zsmem, 1};
    L[k++] = {(void*)fs_ypass_kernel<-1, T>, dim3(p->nx * ntile), dim3(256), ys, 0};
    L[k++] = {(void*)fs_xg_kernel<T>, dim3(p->ny * ntile), dim3(256), xs, 0};
    L[k++] = {(void*)fs_ypass_kernel<1, T>, dim3(p->nx * ntile), dim3(256), ys, 0};
    L[k++] = {zmode == 0 ? (void*)fs_zinv_kernel<0, T> : (void*)fs_zinv_kernel<1, double>, dim3(zl), dim3(256),
              zmode == 0 ? zs : p->zsmem, 0};
  }
  return k;
}

// one matvec / projection in precision T: zfwd<MODE> -> y -> xG -> y^-1 -> zinv<ZMODE>
template <typename T>
static int fs_project(mgk_fs3d_t p, int mode, int zmode, cudaStream_t s) {
  FsArgs a = fs_args(p);
  FsLaunch L[6];
  const int nl = fs_stage_launches<T>(p, mode, zmode, L);
  const double* dbar = p->dbar;
  void* az[] = {&a, (void*)&dbar};
  void* a1[] = {&a};
  for (int k = 0; k < nl; ++k)
    MGK_CUDA(cudaLaunchKernel(L[k].fn, L[k].grid, L[k].block, L[k].args ? az : a1, L[k].smem, s));
  return MGK_OK;
}

static int fs_read_scalars(mgk_fs3d_t p, cudaStream_t s) {
  MGK_CUDA(cudaMemcpyAsync(p->h_sc, p->sc, sizeof(FsScalars), cudaMemcpyDeviceToHost, s));
  MGK_CUDA(cudaStreamSynchronize(s));
  return MGK_OK;
}

// constitutive at F + alpha (x + dbar); results in Ftr/Ptr and the scalars
static int fs_trial(mgk_fs3d_t p, double alpha, bool use_dbar, bool use_x, cudaStream_t s) {
  FsArgs a = fs_args(p);
  fs_constitutive_kernel<<<p->nblk, 256, 0, s>>>(a, alpha, use_dbar ? p->dbar : nullptr, use_x ? 1 : 0);
  fs_constitutive_finalize<<<1, 256, 0, s>>>(a, p->nblk);
  MGK_CUDA(cudaGetLastError());
  return fs_read_scalars(p, s);
}

// accept the trial state: copies (the plane addresses stay fixed, so the
// Krylov graphs stay valid), and the tangent state at the new F
static int fs_accept(mgk_fs3d_t p, cudaStream_t s) {
  MGK_CUDA(cudaMemcpyAsync(p->F, p->Ftr, sizeof(double) * 9 * p->N, cudaMemcpyDeviceToDevice, s));
  MGK_CUDA(cudaMemcpyAsync(p->P, p->Ptr, sizeof(double) * 9 * p->N, cudaMemcpyDeviceToDevice, s));
  return fs_tangent(p, s);
}

// Krylov loop graph for matvec precision T: scalar<2> (norm of the
// right-hand side, sets the loop condition), then while (condition) {matvec,
// alpha, update, beta + decision}.
template <typename T>
static int fs_build_graph(mgk_fs3d_t p, int slot) {
  cudaGraph_t g = nullptr;
  MGK_CUDA(cudaGraphCreate(&g, 0));
  int rc = MGK_OK;
  cudaGraphConditionalHandle h;
  FsArgs a = fs_args(p);
  const int zl = (int)(p->N / p->nz / 2);
  int one = 1, nb = p->nblk;
  auto add = [&](cudaGraph_t gr, cudaGraphNode_t* node, const cudaGraphNode_t* dep, void* fn, dim3 grid, dim3 block,
                 size_t smem, void** args) {
    cudaKernelNodeParams k;
    memset(&k, 0, sizeof(k));
    k.func = fn;
    k.gridDim = grid;
    k.blockDim = block;
    k.sharedMemBytes = (unsigned)smem;
    k.kernelParams = args;
    if (rc == MGK_OK && cudaGraphAddKernelNode(node, gr, dep, dep ? 1 : 0, &k) != cudaSuccess) rc = MGK_CUDA_ERROR;
  };
  if (cudaGraphConditionalHandleCreate(&h, g, 0, cudaGraphCondAssignDefault) != cudaSuccess) rc = MGK_CUDA_ERROR;
  cudaGraphNode_t n0 = nullptr, wn = nullptr;
  void* a_s2[] = {&a, (void*)&zl, &h, &one};
  add(g, &n0, nullptr, (void*)fs_scalar_kernel<2>, dim3(1), dim3(256), 0, a_s2);
  cudaGraph_t body = nullptr;
  if (rc == MGK_OK) {
    alignas(cudaGraphNodeParams) unsigned char raw[sizeof(cudaGraphNodeParams)];
    memset(raw, 0, sizeof(raw));
    cudaGraphNodeParams& cp = *reinterpret_cast<cudaGraphNodeParams*>(raw);
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    if (cudaGraphAddNode(&wn, g, &n0, 1, &cp) != cudaSuccess) rc = MGK_CUDA_ERROR;
    else body = cp.conditional.phGraph_out[0];
  }
  const double* dbar = p->dbar;
  void* a_z[] = {&a, (void*)&dbar};
  void* a_1[] = {&a};
  void* a_s0[] = {&a, (void*)&zl, &h, &one};
  void* a_s1[] = {&a, &nb, &h, &one};
  cudaGraphNode_t kn[6], k6, k7, k8;
  FsLaunch L[6];
  const int nl = fs_stage_launches<T>(p, 0, 0, L);
  for (int k = 0; k < nl; ++k)
    add(body, &kn[k], k ? &kn[k - 1] : nullptr, L[k].fn, L[k].grid, L[k].block, L[k].smem, L[k].args ? a_z : a_1);
  add(body, &k6, &kn[nl - 1], (void*)fs_scalar_kernel<0>, dim3(1), dim3(256), 0, a_s0);
  add(body, &k7, &k6, (void*)fs_update_kernel<T>, dim3(p->nblk), dim3(256), 0, a_1);
  add(body, &k8, &k7, (void*)fs_scalar_kernel<1>, dim3(1), dim3(256), 0, a_s1);
  cudaGraphExec_t x = nullptr;
  if (rc == MGK_OK && cudaGraphInstantiate(&x, g, 0) != cudaSuccess) rc = MGK_CUDA_ERROR;
  if (rc != MGK_OK) {
    cudaGraphDestroy(g);
    cudaGetLastError();
    return rc;
  }
  p->cg_graph[slot] = g;
  p->cg_exec[slot] = x;
  return MGK_OK;
}

// Krylov solve of G:K:dx = r (r holds the right-hand side, x = 0): on the
// device through the graph, or host-driven (one scalar read per iteration)
// when conditional graphs are unavailable.
template <typename T>
static int fs_krylov_run(mgk_fs3d_t p, double tol_CG, int max_cg, cudaStream_t s, int slot, int zl);

template <typename T>
static int fs_krylov(mgk_fs3d_t p, double tol_CG, int max_cg, cudaStream_t s) {
  const int slot = sizeof(T) == 8 ? 0 : 1;
  const int zl = (int)(p->N / p->nz / 2);
  if (sizeof(T) == 4) {
    // FP32 Krylov vectors: r from the FP64 right-hand side, x = 0
    fs_to_f32_kernel<<<p->nblk, 256, 0, s>>>(9 * p->N, p->r, p->r32);
    MGK_CUDA(cudaGetLastError());
    MGK_CUDA(cudaMemsetAsync(p->x32, 0, sizeof(float) * 9 * p->N, s));
  }
  int rc2 = fs_krylov_run<T>(p, tol_CG, max_cg, s, slot, zl);
  if (rc2 == MGK_OK && sizeof(T) == 4) {
    fs_to_f64_kernel<<<p->nblk, 256, 0, s>>>(9 * p->N, p->x32, p->x);
    MGK_CUDA(cudaGetLastError());
  }
  return rc2;
}

template <typename T>
static int fs_krylov_run(mgk_fs3d_t p, double tol_CG, int max_cg, cudaStream_t s, int slot, int zl) {
  if (p->graph_mode < 0) {
    const char* env = getenv("MGK_NO_GRAPH_WHILE");
    p->graph_mode = (env && env[0] == '1') ? 0 : 1;
  }
  if (p->graph_mode == 1 && !p->cg_exec[slot] && fs_build_graph<T>(p, slot) != MGK_OK) p->graph_mode = 0;
  if (p->graph_mode == 1) {
    p->h_dbar[10] = tol_CG * tol_CG;
    p->h_dbar[11] = (double)max_cg;
    MGK_CUDA(cudaMemcpyAsync(&p->sc->tol2, &p->h_dbar[10], 2 * sizeof(double), cudaMemcpyHostToDevice, s));
    MGK_CUDA(cudaGraphLaunch(p->cg_exec[slot], s));
    int rc = fs_read_scalars(p, s);
    if (rc) return rc;
    p->stat_krylov += (int)p->h_sc->kcount;
    if (!isfinite(p->h_sc->rr)) { set_error("mgk_fs3d_step: non-finite Krylov residual"); return MGK_NONFINITE; }
    return MGK_OK;
  }
  FsArgs a = fs_args(p);
  fs_scalar_kernel<2><<<1, 256, 0, s>>>(a, zl, 0, 0);
  MGK_CUDA(cudaGetLastError());
  int rc = fs_read_scalars(p, s);
  if (rc) return rc;
  const double bnorm = sqrt(p->h_sc->bb);
  for (int k = 0; k < max_cg; ++k) {
    if (!(sqrt(p->h_sc->rr) > tol_CG * bnorm)) break;
    rc = fs_project<T>(p, 0, 0, s);
    if (rc) return rc;
    fs_scalar_kernel<0><<<1, 256, 0, s>>>(a, zl, 0, 0);
    fs_update_kernel<T><<<p->nblk, 256, 0, s>>>(a);
    fs_scalar_kernel<1><<<1, 256, 0, s>>>(a, p->nblk, 0, 0);
    MGK_CUDA(cudaGetLastError());
    rc = fs_read_scalars(p, s);
    if (rc) return rc;
    ++p->stat_krylov;
    if (!isfinite(p->h_sc->rr)) { set_error("mgk_fs3d_step: non-finite Krylov residual"); return MGK_NONFINITE; }
  }
  return MGK_OK;
}

// Newton branch (:3046-3119).  F holds F_start on entry, F_curr on exit.
static int fs_newton(mgk_fs3d_t p, const double* F_bar, double tol_NW, double tol_CG, int max_NW, int max_cg,
                     cudaStream_t s) {
  FsArgs a = fs_args(p);
  fs_meanF_kernel<<<p->nblk, 256, 0, s>>>(a);
  fs_meanF_finalize<<<1, 256, 0, s>>>(a, p->nblk);
  MGK_CUDA(cudaGetLastError());
  int rc = fs_read_scalars(p, s);
  if (rc) return rc;
  for (int q = 0; q < 9; ++q) p->h_dbar[q] = F_bar[q] - p->h_sc->meanF[q];
  MGK_CUDA(cudaMemcpyAsync(p->dbar, p->h_dbar, sizeof(double) * 9, cudaMemcpyHostToDevice, s));
  // P, K at F_start
  rc = fs_trial(p, 0.0, false, false, s);
  if (rc) return rc;
  if ((rc = fs_accept(p, s))) return rc;
  for (int it = 0; it < max_NW; ++it) {
    // right-hand side into r (x = 0), always FP64
    rc = fs_project<double>(p, it == 0 ? 1 : 2, 1, s);
    if (rc) return rc;
    rc = p->prec == MGK_MIXED ? fs_krylov<float>(p, tol_CG, max_cg, s) : fs_krylov<double>(p, tol_CG, max_cg, s);
    if (rc) return rc;
    // line search (:3088-3114)
    double alpha = 1.0;
    bool ok = false;
    for (int t = 0; t < 16; ++t) {
      rc = fs_trial(p, alpha, it == 0, true, s);
      if (rc) return rc;
      const FsScalars& S = *p->h_sc;
      if (!(S.minJe > 1e-4) || S.nan != 0) { alpha *= 0.5; continue; }
      ok = true;
      break;
    }
    if (!ok) { set_error("Newton-CG line search failed to find a valid step."); return MGK_NOT_CONVERGED; }
    if ((rc = fs_accept(p, s))) return rc;
    ++p->stat_newton;
    const double res = sqrt(p->h_sc->xx) / (sqrt(std::max(0.0, p->h_sc->FF - p->ff_offset)) + 1e-20);
    if (res < tol_NW && it > 0) return MGK_OK;
  }
  set_error("Newton-CG inner solver did not converge within %d iterations.", max_NW);
  return MGK_NOT_CONVERGED;
}

// Timing hook: mean duration (ms, CUDA events on `stream`) of each kernel
// of one Krylov iteration in the plan's kernel family: [0] z forward (p
// update + K:p + R2C), [1] y pass, [2] x pass with G, [3] inverse y pass,
// [4] z inverse (C2R + p.q), [5] CG update.  fp32 = 1 times the mixed form's
// FP32 kernels.  Runs `reps` iterations on the current state and leaves the
// Krylov vectors in an unspecified state.
extern "C" int mgk_fs3d_profile(mgk_fs3d_t p, int fp32, int reps, float* ms_out, mgk_stream_t stream) {
  MGK_REQUIRE(p && ms_out && reps >= 1 && p->has_material, "mgk_fs3d_profile: bad argument");
  MGK_REQUIRE(!fp32 || p->prec == MGK_MIXED, "mgk_fs3d_profile: fp32 needs a mixed-precision plan");
  cudaStream_t s = (cudaStream_t)stream;
  FsArgs a = fs_args(p);
  FsLaunch L[6];
  const int nl = fp32 ? fs_stage_launches<float>(p, 0, 0, L) : fs_stage_launches<double>(p, 0, 0, L);
  // with a separate tangent-product kernel its time is folded into the z forward entry
  const int first = nl - 5;
  const double* dbar = p->dbar;
  void* az[] = {&a, (void*)&dbar};
  void* a1[] = {&a};
  cudaEvent_t ev[7];
  for (int i = 0; i < 7; ++i) MGK_CUDA(cudaEventCreate(&ev[i]));
  double acc[6] = {0, 0, 0, 0, 0, 0};
  int rc = MGK_OK;
  for (int r = 0; r < reps && rc == MGK_OK; ++r) {
    cudaEventRecord(ev[0], s);
    for (int k = 0; k < nl; ++k) {
      if (cudaLaunchKernel(L[k].fn, L[k].grid, L[k].block, L[k].args ? az : a1, L[k].smem, s) != cudaSuccess)
        rc = MGK_CUDA_ERROR;
      if (k >= first) cudaEventRecord(ev[k - first + 1], s);
    }
    if (fp32) fs_update_kernel<float><<<p->nblk, 256, 0, s>>>(a);
    else fs_update_kernel<double><<<p->nblk, 256, 0, s>>>(a);
    cudaEventRecord(ev[6], s);
    if (cudaEventSynchronize(ev[6]) != cudaSuccess) rc = MGK_CUDA_ERROR;
    for (int k = 0; k < 6; ++k) {
      float ms = 0;
      cudaEventElapsedTime(&ms, ev[k], ev[k + 1]);
      acc[k] += ms;
    }
  }
  for (int i = 0; i < 7; ++i) cudaEventDestroy(ev[i]);
  if (rc != MGK_OK) { cudaGetLastError(); set_error("mgk_fs3d_profile: kernel failure"); return rc; }
  for (int k = 0; k < 6; ++k) ms_out[k] = (float)(acc[k] / reps);
  return MGK_OK;
}

// Autotuner: times one Krylov iteration of each kernel family that can serve
// the plan (warp-line passes when every side is 64/96/128, the CTA-wide
// passes always) on the current state and keeps the faster one.
extern "C" int mgk_fs3d_autotune(mgk_fs3d_t p, int reps, int* chosen, float* best_ms, mgk_stream_t stream) {
  MGK_REQUIRE(p && reps >= 1 && p->has_material, "mgk_fs3d_autotune: bad argument");
  const bool can_fast = fs_fast_len(p->nx) && fs_fast_len(p->ny) && fs_fast_len(p->nz);
  const int fp32 = p->prec == MGK_MIXED ? 1 : 0;
  int best = p->fast;
  float best_t = 0.0f;
  const int cands[2] = {0, 1};
  const int k0 = 0, k1 = can_fast ? 2 : 1;
  for (int k = k0; k < k1; ++k) {
    p->fast = cands[k];
    float ms[6];
    int st = mgk_fs3d_profile(p, fp32, reps, ms, stream);
    if (st) return st;
    float t = 0;
    for (float v : ms) t += v;
    if (k == k0 || t < best_t) { best_t = t; best = cands[k]; }
  }
  p->fast = best;
  fs_drop_graphs(p);
  if (chosen) *chosen = best;
  if (best_ms) *best_ms = best_t;
  return MGK_OK;
}

extern "C" int mgk_fs3d_set_plane_strain(mgk_fs3d_t p, int on) {
  MGK_REQUIRE(p && (!on || p->ny == 1), "mgk_fs3d_set_plane_strain: the plan must be (nx, 1, ny)");
  p->ff_offset = on ? (double)p->N : 0.0;
  return MGK_OK;
}

extern "C" int mgk_fs3d_set_plane_stress(mgk_fs3d_t p, int on) {
  MGK_REQUIRE(p && (!on || p->ny == 1), "mgk_fs3d_set_plane_stress: the plan must be (nx, 1, ny)");
  p->plane_stress = on ? 1 : 0;
  p->ff_offset = on ? (double)p->N : 0.0;
  return MGK_OK;
}

extern "C" int mgk_fs3d_step(mgk_fs3d_t p, const double* F_bar_in, int drv_i, int drv_j, const double* P_target,
                             const int* P_mask, double E_avg, double nu_avg, double tol_NW, double tol_CG, int max_NW,
                             double tol_macro, int max_iter_macro, double* F_bar_out, mgk_fs_info* info,
                             mgk_stream_t stream) {
  MGK_REQUIRE(p && p->has_material && F_bar_in && F_bar_out, "mgk_fs3d_step: bad argument (material set?)");
  MGK_REQUIRE(max_NW >= 1 && max_iter_macro >= 1, "mgk_fs3d_step: iteration caps must be positive");
  cudaStream_t s = (cudaStream_t)stream;
  double Fb[9], tgt[9] = {0};
  int mask[9] = {0};
  for (int q = 0; q < 9; ++q) {
    Fb[q] = F_bar_in[q];
    if (P_target) tgt[q] = P_target[q];
    if (P_mask) mask[q] = P_mask[q] != 0;
  }
  bool any_mask = false;
  for (int q = 0; q < 9; ++q) any_mask |= mask[q] != 0;
  int upd[3] = {0, 0, 0};
  for (int k = 0; k < 3; ++k) upd[k] = mask[4 * k] && !(k == drv_i && k == drv_j);
  bool have_prev = false;
  double prevF[3] = {0, 0, 0}, prevS[3] = {0, 0, 0};
  p->stat_newton = p->stat_krylov = p->stat_macro = 0;
  double max_err = 0.0;
  int rc = MGK_OK;
  for (int it = 0; it < max_iter_macro; ++it) {
    rc = fs_newton(p, Fb, tol_NW, tol_CG, max_NW, 150, s);
    ++p->stat_macro;
    if (rc) break;
    const double* Sm = p->h_sc->sig;
    if (!any_mask) break;
    double err[9] = {0};
    max_err = 0.0;
    for (int q = 0; q < 9; ++q)
      if (mask[q]) { err[q] = tgt[q] - Sm[q]; max_err = std::max(max_err, fabs(err[q])); }
    if (max_err < tol_macro) break;
    const double trerr = err[0] + err[4] + err[8];
    double dF[9];
    for (int q = 0; q < 9; ++q)
      dF[q] = std::min(0.01, std::max(-0.01, (err[q] - ((q % 4 == 0) ? nu_avg * trerr : 0.0)) / E_avg));
    double d_sc[3], Fsc[3], ssc[3];
    for (int k = 0; k < 3; ++k) { d_sc[k] = dF[4 * k]; Fsc[k] = Fb[4 * k]; ssc[k] = Sm[4 * k]; }
    if (have_prev) {
      for (int k = 0; k < 3; ++k) {
        if (!upd[k]) continue;
        const double dh = Fsc[k] - prevF[k];
        const double slope = (ssc[k] - prevS[k]) / dh;
        if (isfinite(slope) && fabs(dh) > 1e-14 && slope > 0.01 * E_avg)
          d_sc[k] = std::min(0.01, std::max(-0.01, err[4 * k] / slope));
      }
    }
    for (int k = 0; k < 3; ++k) { prevF[k] = Fsc[k]; prevS[k] = ssc[k]; }
    have_prev = true;
    for (int k = 0; k < 3; ++k)
      if (upd[k]) Fb[4 * k] += d_sc[k];
    if (it == max_iter_macro - 1) {
      set_error("Outer BC loop did not converge after %d iterations. Final max stress error: %.2e Pa", max_iter_macro,
                max_err);
      rc = MGK_NOT_CONVERGED;
    }
  }
  for (int q = 0; q < 9; ++q) F_bar_out[q] = Fb[q];
  if (info) {
    info->newton_iterations = p->stat_newton;
    info->krylov_iterations = p->stat_krylov;
    info->macro_iterations = p->stat_macro;
    info->status = rc;
    info->max_stress_error = max_err;
    for (int q = 0; q < 9; ++q) info->sig_mean[q] = p->h_sc->sig[q];
  }
  return rc;
}
