// 3D small-strain Lippmann-Schwinger solver (FP64), batched over replicas.
//
// Restates mgkmc/linear_elastic_simulator.py:274-376 (spectral_solver_3d) and
// the 3D Green operator of mgkmc/elasticity.py:70-105, applied on the fly:
//   tau = C:(eps - eps_p) - C0:eps;  eps_new = eps_bar - IFFT(Gamma0 : FFT(tau));
//   diff = ||eps_new - eps|| / (||eps|| + 1e-20).
//
// HBM layout per replica, N = nx*ny*nz (C order, z fastest):
//   mu, lam           2 planes
//   eps[6]            symmetric components xx, yy, zz, yz, xz, xy
//   ep[6]             eigenstrain, symmetric components
//   epf[9]            eigenstrain as given (only when given; output stress)
//   spec[6]           half spectrum [c][x][y][kz], kz < nz/2+1
// The antisymmetric part of eps is uniform after the first iteration and is
// carried as three scalars.
//
// One iteration = four kernels:
//   zline  (CTA per pair of z-lines): C2R along z of the previous spectrum,
//          eps update, diff/norm partials (+ device convergence decision),
//          tau, R2C along z;
//   axis   FFT along y (forward);
//   xgamma FFT along x, eps~^ = -Gamma0_sym : tau^ / N, IFFT along x;
//   axis   IFFT along y.
// Nyquist handling and the device-driven CUDA-graph loop are as in the 2D
// solver (ls2d.cu): Gamma_sym averages Gamma over q and its mirror in the
// Nyquist components, with numpy's fftfreq signs.
#include <math.h>
#include <stddef.h>
#include <stdlib.h>

#include <algorithm>
#include <vector>

#include "common.cuh"
#include "fft.cuh"
#include "tma.cuh"

namespace mgk {

const void* twiddles(int n, int prec);

struct Ls3dRep {
  int nx, ny, nz, nzh, ld, tc;
  int zl_items;      // z-line pairs = nx*ny/2
  int y_items;       // nx * ceil(nzh/tc)
  int x_items;       // ny * ceil(nzh/tc)
  long long N;
  FftLen fx, fy, fz;
  double* mu;
  double* lam;
  double* eps;   // 6 planes
  double* ep;    // 6 planes
  double* epf;   // 9 planes or null
  double2* spec;
  // mixed-precision plans (warp-line kernels only): FP32 copies and tables;
  // the FP32 spectrum reuses `spec`
  float* mu32;
  float* lam32;
  float* eps32;  // 6 planes
  float* ep32;   // 6 planes
  FftLen fx32, fy32, fz32;
  // per call
  const double* init;
  double* out_eps;
  double* out_sig;
  double eb[9];
  double tol;
  int max_iter;
  int zl_first;
  // constitutive law: 0 linear (elasticity.py:62-67); 1 the secant
  // degradation law with magnitude law_a and rate law_b (FP64 plans)
  int law;
  double law_a, law_b;
  // law 3, Landau: v1, v2, v3, g1, g2, g3, g4, capping (0 none, 1 piecewise,
  // 2 smooth), E_cap, tangent ratio, smooth power
  double lp[11];
};

struct Ls3dState {
  double mu0, lam0, Bc, inv2mu0;
  double ebar[6];
  double abar[3];  // (xy - yx)/2, (xz - zx)/2, (yz - zy)/2 of eps_bar
  double extra_d0, extra_n0;
  int iter, done, status, phase_iter;  // done: 0 active, 1 phase 1 finished, 2 finished
  double diff;
  double means[9];
  double out_eps_mean[9];
  double out_sig_mean[9];
};

struct Ls3dCtl {
  unsigned int n_active, decided, still, bodies;
  int any;
  int error;  // a bounded wait gave up (MGK_TIMEOUT)
};

constexpr double kL3Phase1Tol = 2e-6;  // mixed plans: FP32 iterations down to max(tol, this)
constexpr int kL3Phase1Cap = 64;

// symmetric component c -> (i, j): xx yy zz yz xz xy
__device__ __constant__ int kSymI[6] = {0, 1, 2, 1, 0, 0};
__device__ __constant__ int kSymJ[6] = {0, 1, 2, 2, 2, 1};

__device__ __forceinline__ int fftfreq3(int k, int n) { return (k < (n + 1) / 2) ? k : k - n; }

// eps~^ = -Gamma0(n) : tau^ for symmetric tau (3D), n a unit vector.
// t[6] / e[6] in the symmetric order above.
// R = double for the FP64 iterations, float for the FP32 phase of a mixed plan.
template <typename R>
__device__ __forceinline__ void gamma3d_apply_t(const C_t<R>* t, R n0, R n1, R n2, R inv2mu0, R Bc, C_t<R>* e) {
  constexpr int kI[6] = {0, 1, 2, 1, 0, 0}, kJ[6] = {0, 1, 2, 2, 2, 1};
  const R n[3] = {n0, n1, n2};
  // full symmetric tau as 3x3 of complex
  C_t<R> T[3][3];
  T[0][0] = t[0]; T[1][1] = t[1]; T[2][2] = t[2];
  T[1][2] = T[2][1] = t[3];
  T[0][2] = T[2][0] = t[4];
  T[0][1] = T[1][0] = t[5];
  C_t<R> tn[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    tn[i].x = T[i][0].x * n[0] + T[i][1].x * n[1] + T[i][2].x * n[2];
    tn[i].y = T[i][0].y * n[0] + T[i][1].y * n[1] + T[i][2].y * n[2];
  }
  C_t<R> ntn;
  ntn.x = tn[0].x * n[0] + tn[1].x * n[1] + tn[2].x * n[2];
  ntn.y = tn[0].y * n[0] + tn[1].y * n[1] + tn[2].y * n[2];
#pragma unroll
  for (int c = 0; c < 6; ++c) {
    const int k = kI[c], h = kJ[c];
    e[c].x = -(inv2mu0 * (n[h] * tn[k].x + n[k] * tn[h].x) - Bc * n[k] * n[h] * ntn.x);
    e[c].y = -(inv2mu0 * (n[h] * tn[k].y + n[k] * tn[h].y) - Bc * n[k] * n[h] * ntn.y);
  }
}
__device__ __forceinline__ void gamma3d_apply(const double2* t, double n0, double n1, double n2, double inv2mu0,
                                              double Bc, double2* e) {
  gamma3d_apply_t<double>(t, n0, n1, n2, inv2mu0, Bc, e);
}

// -------------------------------------------------------------- kernels ---

// Secant shear modulus mu (1 - d (1 - exp(-k eq))) (elasticity.py:703-728) at
// the von Mises equivalent strain sqrt(2/3 e':e') of the elastic strain
// (elasticity.py:665-700) given by its symmetric components; each pair of
// shear entries sums to twice the symmetric one.
// 3D Landau small-strain stress (elasticity.py:811-857) of the symmetric
// elastic strain a = (xx, yy, zz, yz, xz, xy), with the strain capping of
// elasticity.py:297-334: deviator scaled by f above the cap E_cap (piecewise)
// or by the tanh profile (smooth), plus 2 (ratio mu) (a - capped) w.
// sigma = (lam I1 + v1/2 I1^2 + v2 I2 + g1/6 I1^3 + g2 I1 I2 + 4/3 g3 I3) I
//       + 2 (mu + v2 I1 + g2/2 I1^2 + g4 I2) e + 4 (v3 + g3 I1) e^2.
__device__ __forceinline__ void landau_sigma3(double mu, double lam, const double* a, const double* __restrict__ lp,
                                              double* sg) {
  const double v1 = lp[0], v2 = lp[1], v3 = lp[2], g1 = lp[3], g2 = lp[4], g3 = lp[5], g4 = lp[6];
  const int cap = (int)lp[7];
  double c[6];
  for (int q = 0; q < 6; ++q) c[q] = a[q];
  double w = 0.0;
  if (cap) {
    const double I1a = a[0] + a[1] + a[2];
    const double m3 = (1.0 / 3.0) * I1a;
    const double d0 = a[0] - m3, d1 = a[1] - m3, d2 = a[2] - m3;
    const double dd = d0 * d0 + d1 * d1 + d2 * d2 + 2.0 * (a[3] * a[3] + a[4] * a[4] + a[5] * a[5]);
    const double Eeq = sqrt(fmax(0.0, (2.0 / 3.0) * dd));
    const double Ecap = lp[8];
    double f = 1.0;
    if (cap == 2) {
      const double pw = lp[10];
      if (Eeq > 1e-12) f = (Ecap / Eeq) * pow(tanh(fmin(100.0, pow(Eeq / Ecap, pw))), 1.0 / pw);
      const double t = tanh(fmin(100.0, pow(Eeq / Ecap, pw)));
      w = t * t;
    } else if (Eeq > Ecap) {
      f = Ecap / Eeq;
      w = 1.0;
    }
    c[0] = d0 * f + m3;
    c[1] = d1 * f + m3;
    c[2] = d2 * f + m3;
    c[3] = a[3] * f;
    c[4] = a[4] * f;
    c[5] = a[5] * f;
  }
  // e^2 of the symmetric tensor [[xx, xy, xz], [xy, yy, yz], [xz, yz, zz]]
  const double xx = c[0], yy = c[1], zz = c[2], yz = c[3], xz = c[4], xy = c[5];
  double e2[6];
  e2[0] = xx * xx + xy * xy + xz * xz;
  e2[1] = xy * xy + yy * yy + yz * yz;
  e2[2] = xz * xz + yz * yz + zz * zz;
  e2[3] = xy * xz + yy * yz + yz * zz;
  e2[4] = xx * xz + xy * yz + xz * zz;
  e2[5] = xx * xy + xy * yy + xz * yz;
  const double I1 = xx + yy + zz;
  const double I2 = e2[0] + e2[1] + e2[2];
  const double I3 = (e2[0] * xx + e2[5] * xy + e2[4] * xz) + (e2[5] * xy + e2[1] * yy + e2[3] * yz) +
                    (e2[4] * xz + e2[3] * yz + e2[2] * zz);
  const double cI = lam * I1 + 0.5 * v1 * (I1 * I1) + v2 * I2 + (1.0 / 6.0) * g1 * (I1 * I1 * I1) + g2 * I1 * I2 +
                    (4.0 / 3.0) * g3 * I3;
  const double ce = 2.0 * (mu + v2 * I1 + 0.5 * g2 * (I1 * I1) + g4 * I2);
  const double ce2 = 4.0 * (v3 + g3 * I1);
  for (int q = 0; q < 6; ++q) sg[q] = (q < 3 ? cI : 0.0) + ce * c[q] + ce2 * e2[q];
  if (cap) {
    const double r = 2.0 * (lp[9] * mu) * w;
    for (int q = 0; q < 6; ++q) sg[q] += r * (a[q] - c[q]);
  }
}

__device__ __forceinline__ double secant_mu3(double m, double xx, double yy, double zz, double yz, double xz,
                                             double xy, double d, double k) {
  const double tr3 = (xx + yy + zz) / 3.0;
  const double a = xx - tr3, b = yy - tr3, c = zz - tr3;
  const double s1 = 2.0 * xy, s2 = 2.0 * xz, s3 = 2.0 * yz;
  const double eq = sqrt((2.0 / 3.0) * (a * a + b * b + c * c + 0.5 * (s1 * s1 + s2 * s2 + s3 * s3)));
  return m * (1.0 - d * (1.0 - exp(-k * eq)));
}

__global__ void ls3d_material_kernel(const Ls3dRep* reps, int rep, const double* __restrict__ E,
                                     const double* __restrict__ nu, const double* __restrict__ epsp,
                                     int set_moduli, double* partials) {
  __shared__ double red[32];
  const Ls3dRep& R = reps[rep];
  const long long N = R.N;
  double sE = 0, sn = 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N;
       i += (long long)gridDim.x * blockDim.x) {
    if (set_moduli) {
      // elasticity.py:55-59 (set_moduli 1); set_moduli 2: E holds lambda and
      // nu holds mu, as the secant solver takes them
      const double e = E[i], v = nu[i];
      R.mu[i] = set_moduli == 2 ? v : e / (2 * (1 + v));
      R.lam[i] = set_moduli == 2 ? e : e * v / ((1 + v) * (1 - 2 * v));
      if (R.mu32) { R.mu32[i] = (float)R.mu[i]; R.lam32[i] = (float)R.lam[i]; }
      sE += e;
      sn += v;
    }
    double p[9];
    for (int q = 0; q < 9; ++q) p[q] = epsp ? epsp[9 * i + q] : 0.0;
    for (int c = 0; c < 6; ++c) {
      const int a = 3 * kSymI[c] + kSymJ[c], b = 3 * kSymJ[c] + kSymI[c];
      R.ep[c * N + i] = (p[a] == p[b]) ? p[a] : 0.5 * (p[a] + p[b]);
      if (R.ep32) R.ep32[c * N + i] = (float)R.ep[c * N + i];
    }
    if (R.epf)
      for (int q = 0; q < 9; ++q) R.epf[q * N + i] = p[q];
  }
  if (set_moduli) {
    double a = block_sum(sE, red);
    double b = block_sum(sn, red);
    if (threadIdx.x == 0) { partials[2 * blockIdx.x] = a; partials[2 * blockIdx.x + 1] = b; }
  }
}

// reference medium from the means of E and nu (linear_elastic_simulator.py:
// 284-289), or of lambda and mu (lame_in; the secant solver, :783-784)
__global__ void ls3d_medium_kernel(const Ls3dRep* reps, Ls3dState* st, int rep, const double* partials, int nb,
                                   int lame_in) {
  __shared__ double red[32];
  double a = 0, b = 0;
  for (int i = threadIdx.x; i < nb; i += blockDim.x) { a += partials[2 * i]; b += partials[2 * i + 1]; }
  a = block_sum(a, red);
  b = block_sum(b, red);
  if (threadIdx.x == 0) {
    const double N = (double)reps[rep].N;
    const double E = a / N, v = b / N;
    const double mu0 = lame_in ? v : E / (2 * (1 + v));
    const double lam0 = lame_in ? E : E * v / ((1 + v) * (1 - 2 * v));
    Ls3dState& S = st[rep];
    S.mu0 = mu0;
    S.lam0 = lam0;
    S.Bc = (lam0 + mu0) / (mu0 * (lam0 + 2 * mu0));
    S.inv2mu0 = 1.0 / (2 * mu0);
  }
}

// per-CTA partials of the 9 components of the warm-start field; grid (G, nsel)
__global__ void ls3d_means_kernel(const Ls3dRep* reps, const int* sel, double* partials) {
  __shared__ double red[32];
  const Ls3dRep& R = reps[sel[blockIdx.y]];
  if (!R.init) return;
  double s[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < R.N;
       i += (long long)gridDim.x * blockDim.x)
    for (int q = 0; q < 9; ++q) s[q] += R.init[9 * i + q];
  for (int q = 0; q < 9; ++q) {
    double t = block_sum(s[q], red);
    if (threadIdx.x == 0) partials[((size_t)blockIdx.y * gridDim.x + blockIdx.x) * 18 + q] = t;
  }
}

// fixed-order sums (stride 18 per CTA slot); mode 0: means of every replica,
// 1: means for warm-started replicas, 2: plain sums for warm-started replicas
__global__ void ls3d_finalize_kernel(const Ls3dRep* reps, Ls3dState* st, const int* sel, const double* partials,
                                     int G, int K, int off, int mode) {
  __shared__ double red[32];
  const int r = sel[blockIdx.x];
  if (mode && !reps[r].init) return;
  const double scale = mode == 2 ? 1.0 : 1.0 / (double)reps[r].N;
  double* out = reinterpret_cast<double*>(reinterpret_cast<char*>(&st[r]) + off);
  for (int q = 0; q < K; ++q) {
    double a = 0;
    for (int i = threadIdx.x; i < G; i += blockDim.x) a += partials[((size_t)blockIdx.x * G + i) * 18 + q];
    a = block_sum(a, red);
    if (threadIdx.x == 0) out[q] = a * scale;
  }
}

// initial field (linear_elastic_simulator.py:302-313); grid (G, nsel)
__global__ void ls3d_begin_kernel(const Ls3dRep* reps, Ls3dState* st, const int* sel, double* partials) {
  __shared__ double red[32];
  const int r = sel[blockIdx.y];
  const Ls3dRep& R = reps[r];
  Ls3dState& S = st[r];
  const long long N = R.N;
  const double* eb = R.eb;
  double ab[3] = {0.5 * (eb[1] - eb[3]), 0.5 * (eb[2] - eb[6]), 0.5 * (eb[5] - eb[7])};
  double sb[6];
  for (int c = 0; c < 6; ++c) {
    const int a = 3 * kSymI[c] + kSymJ[c], b = 3 * kSymJ[c] + kSymI[c];
    sb[c] = (eb[a] == eb[b]) ? eb[a] : 0.5 * (eb[a] + eb[b]);
  }
  double d2 = 0, n2 = 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N;
       i += (long long)gridDim.x * blockDim.x) {
    if (R.init) {
      double v[9];
      for (int q = 0; q < 9; ++q) v[q] = R.init[9 * i + q] + (eb[q] - S.means[q]);
      for (int c = 0; c < 6; ++c) {
        const int a = 3 * kSymI[c] + kSymJ[c], b = 3 * kSymJ[c] + kSymI[c];
        R.eps[c * N + i] = (v[a] == v[b]) ? v[a] : 0.5 * (v[a] + v[b]);
        if (R.eps32) R.eps32[c * N + i] = (float)R.eps[c * N + i];
      }
      const double a0[3] = {0.5 * (v[1] - v[3]), 0.5 * (v[2] - v[6]), 0.5 * (v[5] - v[7])};
      for (int q = 0; q < 3; ++q) {
        d2 += 2 * (ab[q] - a0[q]) * (ab[q] - a0[q]);
        n2 += 2 * a0[q] * a0[q];
      }
    } else {
      for (int c = 0; c < 6; ++c) {
        R.eps[c * N + i] = sb[c];
        if (R.eps32) R.eps32[c * N + i] = (float)sb[c];
      }
    }
  }
  if (R.init) {
    d2 = block_sum(d2, red);
    n2 = block_sum(n2, red);
    if (threadIdx.x == 0) {
      partials[((size_t)blockIdx.y * gridDim.x + blockIdx.x) * 18 + 0] = d2;
      partials[((size_t)blockIdx.y * gridDim.x + blockIdx.x) * 18 + 1] = n2;
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    for (int c = 0; c < 6; ++c) S.ebar[c] = sb[c];
    for (int q = 0; q < 3; ++q) S.abar[q] = ab[q];
    S.iter = 0;
    S.phase_iter = 0;
    S.done = R.max_iter <= 0 ? 2 : 0;
    S.status = MGK_OK;
    S.diff = 0;
    if (!R.init) {
      S.extra_d0 = 0;
      S.extra_n0 = 2.0 * (double)N * (ab[0] * ab[0] + ab[1] * ab[1] + ab[2] * ab[2]);
    }
  }
}

// Partial sums of this z-line item, and (last item of the replica) the
// fixed-order reduction, the convergence decision and the loop condition.
template <bool FINAL>
__device__ void ls3d_decide(const Ls3dRep& R, Ls3dState& S, int r, int item, double d2, double n2,
                            double* partials, unsigned int* rep_counter, Ls3dCtl* ctl,
                            cudaGraphConditionalHandle cond, int use_cond, int guard_cap, double* red,
                            int* s_last_p) {
  int& s_last = *s_last_p;
  const long long N = R.N;
  d2 = block_sum(d2, red);
  n2 = block_sum(n2, red);
  if (threadIdx.x == 0) {
    partials[2 * item] = d2;
    partials[2 * item + 1] = n2;
    __threadfence();
    const unsigned int t = atomicInc(&rep_counter[r], (unsigned int)R.zl_items - 1);
    s_last = (t == (unsigned int)R.zl_items - 1);
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  double a = 0, b = 0;
  for (int i = threadIdx.x; i < R.zl_items; i += blockDim.x) {
    a += __ldcg(&partials[2 * (R.zl_first + i)]);
    b += __ldcg(&partials[2 * (R.zl_first + i) + 1]);
  }
  a = block_sum(a, red);
  b = block_sum(b, red);
  if (threadIdx.x != 0) return;
  if (S.iter == 0) { a += S.extra_d0; b += S.extra_n0; }
  else b += 2.0 * (double)N * (S.abar[0] * S.abar[0] + S.abar[1] * S.abar[1] + S.abar[2] * S.abar[2]);
  const double diff = sqrt(a) / (sqrt(b) + 1e-20);
  S.diff = diff;
  S.iter += 1;
  S.phase_iter += 1;
  int keep = 0;
  if (!isfinite(diff)) { S.done = 2; S.status = MGK_NONFINITE; }
  else if (FINAL) {
    if (diff < R.tol) { S.done = 2; S.status = MGK_OK; }
    else if (S.iter >= R.max_iter) { S.done = 2; S.status = MGK_NOT_CONVERGED; }
    else keep = 1;
  } else {
    const double tol1 = R.tol > kL3Phase1Tol ? R.tol : kL3Phase1Tol;
    if (S.iter >= R.max_iter) { S.done = 2; S.status = diff < R.tol ? MGK_OK : MGK_NOT_CONVERGED; }
    else if (diff < tol1 || S.phase_iter >= kL3Phase1Cap) S.done = 1;
    else keep = 1;
  }
  const unsigned int n_act = ctl->n_active;
  if (keep) atomicAdd(&ctl->still, 1u);
  __threadfence();
  const unsigned int dcount = atomicAdd(&ctl->decided, 1u);
  if (dcount == n_act - 1) {
    __threadfence();
    const unsigned int still = atomicExch(&ctl->still, 0u);
    ctl->decided = 0;
    ctl->n_active = still;
    const bool go = still > 0 && atomicAdd(&ctl->bodies, 0u) <= (unsigned int)guard_cap;
    ctl->any = go ? 1 : 0;
    if (use_cond) cudaGraphSetConditional(cond, go ? 1u : 0u);
  }
}

// z-line kernel: pairs of z-lines (flattened (x, y) index 2p, 2p+1)
template <bool IN_SPEC>
__global__ void __launch_bounds__(256) ls3d_zline_kernel(const Ls3dRep* __restrict__ reps, Ls3dState* st,
                                                        const int* __restrict__ map, const int* __restrict__ loc,
                                                        double* partials, unsigned int* rep_counter, Ls3dCtl* ctl,
                                                        cudaGraphConditionalHandle cond, int use_cond,
                                                        int guard_cap) {
  using C = double2;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ double red[32];
  __shared__ int s_last;
  const int item = blockIdx.x;
  const int r = map[item];
  const Ls3dRep& R = reps[r];
  Ls3dState& S = st[r];
  if (IN_SPEC && use_cond && item == 0 && threadIdx.x == 0) {
    const unsigned int b = atomicAdd(&ctl->bodies, 1u) + 1u;
    if (ctl->n_active == 0 || b > (unsigned int)guard_cap || *(volatile int*)&ctl->error != 0) {
      ctl->any = 0;
      cudaGraphSetConditional(cond, 0u);
    }
  }
  if (S.done != 0) return;
  const int nz = R.nz, nzh = R.nzh, ld = R.ld;
  const long long N = R.N;
  const long long l0 = 2LL * loc[item];  // first line (flattened x*ny + y)
  const long long plane = (long long)R.nx * R.ny * ld;  // complex elements per component
  C* bufA = reinterpret_cast<C*>(smem_raw);
  C* bufB = bufA + 6 * nz;
  C* spec = R.spec;
  double d2 = 0, n2 = 0;
  C* cur = bufA;
  if (IN_SPEC) {
    const int tot = 6 * nz;
    for (int e = threadIdx.x; e < tot; e += blockDim.x) {
      const int c = e / nz, k = e - c * nz;
      const int ks = (2 * k <= nz) ? k : nz - k;
      const C* ra = spec + c * plane + l0 * ld;
      C a = ra[ks], b = ra[ld + ks];
      C z;
      if (2 * k <= nz) {
        if (k == 0 || 2 * k == nz) { a.y = 0; b.y = 0; }
        z = make_double2(a.x - b.y, a.y + b.x);
      } else {
        z = make_double2(a.x + b.y, b.x - a.y);
      }
      bufA[e] = z;
    }
    __syncthreads();
    cur = fft_any<+1>(bufA, bufB, 6, nz, R.fz);
  }
  C* out = (IN_SPEC && cur == bufA) ? bufB : bufA;
  const double mu0 = S.mu0, lam0 = S.lam0;
  for (int z = threadIdx.x; z < nz; z += blockDim.x) {
    double tr[2][6];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const long long i = (l0 + h) * nz + z;
      double e[6];
#pragma unroll
      for (int c = 0; c < 6; ++c) {
        const double o = R.eps[c * N + i];
        if (IN_SPEC) {
          const C zz = cur[c * nz + z];
          const double nw = S.ebar[c] + (h == 0 ? zz.x : zz.y);
          const double dd = nw - o;
          const double w = c < 3 ? 1.0 : 2.0;
          d2 += w * dd * dd;
          n2 += w * o * o;
          R.eps[c * N + i] = nw;
          e[c] = nw;
        } else {
          e[c] = o;
        }
      }
      double m = R.mu[i];
      const double l = R.lam[i];
      double d[6];
#pragma unroll
      for (int c = 0; c < 6; ++c) d[c] = e[c] - R.ep[c * N + i];
      if (R.law == 1) m = secant_mu3(m, d[0], d[1], d[2], d[3], d[4], d[5], R.law_a, R.law_b);
      const double trd = d[0] + d[1] + d[2], tre = e[0] + e[1] + e[2];
      if (R.law == 3) {
        double sg[6];
        landau_sigma3(m, l, d, R.lp, sg);
#pragma unroll
        for (int c = 0; c < 3; ++c) tr[h][c] = sg[c] - (2 * mu0 * e[c] + lam0 * tre);
#pragma unroll
        for (int c = 3; c < 6; ++c) tr[h][c] = sg[c] - 2 * mu0 * e[c];
      } else {
#pragma unroll
        for (int c = 0; c < 3; ++c) tr[h][c] = (2 * m * d[c] + l * trd) - (2 * mu0 * e[c] + lam0 * tre);
#pragma unroll
        for (int c = 3; c < 6; ++c) tr[h][c] = 2 * m * d[c] - 2 * mu0 * e[c];
      }
    }
#pragma unroll
    for (int c = 0; c < 6; ++c) out[c * nz + z] = make_double2(tr[0][c], tr[1][c]);
  }
  __syncthreads();
  C* scratch = (out == bufA) ? bufB : bufA;
  C* Z = fft_any<-1>(out, scratch, 6, nz, R.fz);
  for (int e = threadIdx.x; e < 6 * nzh; e += blockDim.x) {
    const int c = e / nzh, k = e - c * nzh;
    const C z = Z[c * nz + k];
    const C w = Z[c * nz + (k == 0 ? 0 : nz - k)];
    C* ra = spec + c * plane + l0 * ld;
    ra[k] = make_double2(0.5 * (z.x + w.x), 0.5 * (z.y - w.y));
    ra[ld + k] = make_double2(0.5 * (z.y + w.y), -0.5 * (z.x - w.x));
  }
  if (!IN_SPEC) return;
  ls3d_decide<true>(R, S, r, item, d2, n2, partials, rep_counter, ctl, cond, use_cond, guard_cap, red, &s_last);
}

// Strided-axis pass over tiles of tc consecutive kz columns.
// AXIS = 1: FFT along y (SIGN given); AXIS = 0: FFT along x, Gamma0_sym,
// IFFT along x.
template <int AXIS, int SIGN>
__global__ void __launch_bounds__(256) ls3d_axis_kernel(const Ls3dRep* __restrict__ reps,
                                                       const Ls3dState* __restrict__ st,
                                                       const int* __restrict__ map, const int* __restrict__ loc) {
  using C = double2;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int item = blockIdx.x;
  const int r = map[item];
  const Ls3dRep& R = reps[r];
  const Ls3dState& S = st[r];
  if (S.done != 0) return;
  const int nx = R.nx, ny = R.ny, nz = R.nz, nzh = R.nzh, ld = R.ld, tc = R.tc;
  const int ntile = (nzh + tc - 1) / tc;
  const int o = loc[item] / ntile;          // x (AXIS 1) or y (AXIS 0)
  const int k0 = (loc[item] - o * ntile) * tc;
  const int tcw = min(tc, nzh - k0);
  const int n = AXIS == 1 ? ny : nx;
  const FftLen& f = AXIS == 1 ? R.fy : R.fx;
  const long long plane = (long long)nx * ny * ld;
  const long long lstride = AXIS == 1 ? ld : (long long)ny * ld;
  const long long obase = AXIS == 1 ? (long long)o * ny * ld : (long long)o * ld;
  C* bufA = reinterpret_cast<C*>(smem_raw);
  C* bufB = bufA + 6 * tc * n;
  C* spec = R.spec;
  const int tot = 6 * tcw * n;
  for (int e0 = threadIdx.x; e0 < tot; e0 += 4 * blockDim.x) {
    C v[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int e = e0 + u * blockDim.x;
      if (e < tot) {
        const int c = e / (tcw * n), rem = e - c * tcw * n, j = rem / tcw, t = rem - j * tcw;
        v[u] = spec[c * plane + obase + j * lstride + k0 + t];
      }
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int e = e0 + u * blockDim.x;
      if (e < tot) {
        const int c = e / (tcw * n), rem = e - c * tcw * n, j = rem / tcw, t = rem - j * tcw;
        bufA[(c * tc + t) * n + j] = v[u];
      }
    }
  }
  __syncthreads();
  C* F;
  if (AXIS == 1) {
    F = fft_any<SIGN>(bufA, bufB, 6 * tc, n, f);
  } else {
    C* G = fft_any<-1>(bufA, bufB, 6 * tc, n, f);
    const double scale = 1.0 / (double)R.N;
    const int ky = o;
    const double uy = (double)fftfreq3(ky, ny) / ny;
    const bool nqy = (ny & 1) == 0 && 2 * ky == ny;
    for (int e = threadIdx.x; e < tcw * n; e += blockDim.x) {
      const int t = e / n, kx = e - t * n;
      const int kz = k0 + t;
      C tv[6], ev[6];
      for (int c = 0; c < 6; ++c) tv[c] = G[(c * tc + t) * n + kx];
      if (kx == 0 && ky == 0 && kz == 0) {
        for (int c = 0; c < 6; ++c) G[(c * tc + t) * n + kx] = make_double2(0.0, 0.0);
        continue;
      }
      const double ux = (double)fftfreq3(kx, nx) / nx, uz = (double)fftfreq3(kz, nz) / nz;
      const double inv = 1.0 / sqrt(ux * ux + uy * uy + uz * uz);
      const double n0 = ux * inv, n1 = uy * inv, n2 = uz * inv;
      gamma3d_apply(tv, n0, n1, n2, S.inv2mu0, S.Bc, ev);
      const bool nqx = (nx & 1) == 0 && 2 * kx == nx, nqz = (nz & 1) == 0 && 2 * kz == nz;
      if (nqx || nqy || nqz) {
        C fv[6];
        gamma3d_apply(tv, nqx ? -n0 : n0, nqy ? -n1 : n1, nqz ? -n2 : n2, S.inv2mu0, S.Bc, fv);
        for (int c = 0; c < 6; ++c) ev[c] = make_double2(0.5 * (ev[c].x + fv[c].x), 0.5 * (ev[c].y + fv[c].y));
      }
      for (int c = 0; c < 6; ++c) G[(c * tc + t) * n + kx] = make_double2(ev[c].x * scale, ev[c].y * scale);
    }
    __syncthreads();
    C* H = (G == bufA) ? bufB : bufA;
    F = fft_any<+1>(G, H, 6 * tc, n, f);
  }
  for (int e = threadIdx.x; e < tot; e += blockDim.x) {
    const int c = e / (tcw * n), rem = e - c * tcw * n, j = rem / tcw, t = rem - j * tcw;
    spec[c * plane + obase + j * lstride + k0 + t] = F[(c * tc + t) * n + j];
  }
}

// --------------------------------------------- warp-line iteration kernels ---
// The same iteration for replicas whose sides are all 64, 96 or 128:
//   z-line kernel: CTA of 3 warps per pair of z-lines; one elected thread
//     stages the pair's eps (6), mu, lambda and eps_p (6) lines in shared
//     memory with bulk copies while warp w inverts components 2w, 2w+1 of the
//     spectrum; after one CTA barrier every thread updates its voxels and
//     builds tau; warp w transforms and stores its two components.
//   axis kernels: per tile of kL3Tile kz columns at one x (y passes) or one y
//     (x pass with Gamma0_sym between the transforms), warp c owns component
//     c's lines; the x pass CTA holds all 6 components, an FP64 y pass CTA 3.
constexpr int kL3Tile = 4;

template <typename T> struct L3F;
template <> struct L3F<double> {
  static __device__ __forceinline__ double* eps(const Ls3dRep& R) { return R.eps; }
  static __device__ __forceinline__ const double* ep(const Ls3dRep& R) { return R.ep; }
  static __device__ __forceinline__ const double* mu(const Ls3dRep& R) { return R.mu; }
  static __device__ __forceinline__ const double* lam(const Ls3dRep& R) { return R.lam; }
  static __device__ __forceinline__ double2* spec(const Ls3dRep& R) { return R.spec; }
  static __device__ __forceinline__ const FftLen& fx(const Ls3dRep& R) { return R.fx; }
  static __device__ __forceinline__ const FftLen& fy(const Ls3dRep& R) { return R.fy; }
  static __device__ __forceinline__ const FftLen& fz(const Ls3dRep& R) { return R.fz; }
};
template <> struct L3F<float> {
  static __device__ __forceinline__ float* eps(const Ls3dRep& R) { return R.eps32; }
  static __device__ __forceinline__ const float* ep(const Ls3dRep& R) { return R.ep32; }
  static __device__ __forceinline__ const float* mu(const Ls3dRep& R) { return R.mu32; }
  static __device__ __forceinline__ const float* lam(const Ls3dRep& R) { return R.lam32; }
  static __device__ __forceinline__ float2* spec(const Ls3dRep& R) { return reinterpret_cast<float2*>(R.spec); }
  static __device__ __forceinline__ const FftLen& fx(const Ls3dRep& R) { return R.fx32; }
  static __device__ __forceinline__ const FftLen& fy(const Ls3dRep& R) { return R.fy32; }
  static __device__ __forceinline__ const FftLen& fz(const Ls3dRep& R) { return R.fz32; }
};
__host__ __device__ constexpr bool ls3_fast_len(int n) { return n == 64 || n == 96 || n == 128; }
__host__ __device__ constexpr int ls3_pl(int n, int csz) { return csz == 16 ? n + n / 8 + 1 : ((n + n / 16 + 2) & ~1); }
__host__ __device__ constexpr int ls3_zl_smem(int nz, int csz) {
  return ((6 * ls3_pl(nz, csz) * csz + 127) / 128) * 128 + 14 * 2 * nz * (csz / 2);
}
__host__ __device__ constexpr int ls3_ax_smem(int n, int csz) { return 6 * kL3Tile * ls3_pl(n, csz) * csz; }

template <typename T, bool IN_SPEC, bool FINAL, int NZ, int LAW>
__device__ __forceinline__ void ls3_zline_body(const Ls3dRep& R, Ls3dState& S, int item, int r, long long l0,
                                               double* partials, unsigned int* rep_counter, Ls3dCtl* ctl,
                                               cudaGraphConditionalHandle cond, int use_cond, int guard_cap,
                                               unsigned char* smem, uint64_t* bar, double* red, int* s_last) {
  using C = C_t<T>;
  constexpr int PL = padded_len<C>(NZ);
  constexpr int NZH = NZ / 2 + 1;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int ld = R.ld;
  const long long N = R.N;
  const long long plane = (long long)R.nx * R.ny * ld;
  C* lines = reinterpret_cast<C*>(smem);
  T* stg = reinterpret_cast<T*>(smem + ((6 * PL * (int)sizeof(C) + 127) / 128) * 128);
  T* eps = L3F<T>::eps(R);
  const T* ep = L3F<T>::ep(R);
  C* spec = L3F<T>::spec(R);
  constexpr uint32_t rb = 2u * NZ * sizeof(T);
  if (threadIdx.x == 0) {
    fence_proxy_async_smem();
    mbar_arrive_expect_tx(bar, 14u * rb);
#pragma unroll
    for (int c = 0; c < 6; ++c) bulk_g2s(stg + c * 2 * NZ, eps + c * N + l0 * NZ, rb, bar);
    bulk_g2s(stg + 12 * NZ, L3F<T>::mu(R) + l0 * NZ, rb, bar);
    bulk_g2s(stg + 14 * NZ, L3F<T>::lam(R) + l0 * NZ, rb, bar);
#pragma unroll
    for (int c = 0; c < 6; ++c) bulk_g2s(stg + (16 + 2 * c) * NZ, ep + c * N + l0 * NZ, rb, bar);
  }
  const C* tw = reinterpret_cast<const C*>(L3F<T>::fz(R).tw);
  C* lw = lines + 2 * warp * PL;
  if (IN_SPEC) {
    constexpr int U = (NZH + 31) / 32;
    for (int cc = 0; cc < 2; ++cc) {
      const int c = 2 * warp + cc;
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
          C a = av[u], b = bv[u];
          if (k == 0 || 2 * k == NZ) { a.y = 0; b.y = 0; }
          ln[pidx<C>(k)] = mk<C>(a.x - b.y, a.y + b.x);
          if (k > 0 && 2 * k < NZ) ln[pidx<C>(NZ - k)] = mk<C>(a.x + b.y, b.x - a.y);
        }
      }
    }
    __syncwarp();
    warp_fft<NZ, +1, 2>(lw, PL, tw, lane);
  }
  const bool ok = mbar_wait(bar, 0);
  if (!__syncthreads_and(ok ? 1 : 0)) {
    if (threadIdx.x == 0) { ctl->error = 1; ctl->any = 0; }
    return;
  }
  const double mu0 = S.mu0, lam0 = S.lam0;
  double d2 = 0, n2 = 0;
  for (int z = threadIdx.x; z < NZ; z += 96) {
    const int pz = pidx<C>(z);
    C zz[6];
    if (IN_SPEC) {
#pragma unroll
      for (int c = 0; c < 6; ++c) zz[c] = lines[c * PL + pz];
    }
    T tr[2][6];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int j = h * NZ + z;
      const long long i = (l0 + h) * NZ + z;
      double e[6];
#pragma unroll
      for (int c = 0; c < 6; ++c) {
        const double o = (double)stg[c * 2 * NZ + j];
        if (IN_SPEC) {
          const double nw = S.ebar[c] + (double)(h == 0 ? zz[c].x : zz[c].y);
          const double dd = nw - o;
          const double w = c < 3 ? 1.0 : 2.0;
          d2 += w * dd * dd;
          n2 += w * o * o;
          eps[c * N + i] = (T)nw;
          e[c] = nw;
        } else {
          e[c] = o;
        }
      }
      double m = (double)stg[12 * NZ + j];
      const double l = (double)stg[14 * NZ + j];
      double d[6];
#pragma unroll
      for (int c = 0; c < 6; ++c) d[c] = e[c] - (double)stg[(16 + 2 * c) * NZ + j];
      if constexpr (LAW == 1) m = secant_mu3(m, d[0], d[1], d[2], d[3], d[4], d[5], R.law_a, R.law_b);
      const double trd = d[0] + d[1] + d[2], tre = e[0] + e[1] + e[2];
      if constexpr (LAW == 3) {
        double sg[6];
        landau_sigma3(m, l, d, R.lp, sg);
#pragma unroll
        for (int c = 0; c < 3; ++c) tr[h][c] = (T)(sg[c] - (2 * mu0 * e[c] + lam0 * tre));
#pragma unroll
        for (int c = 3; c < 6; ++c) tr[h][c] = (T)(sg[c] - 2 * mu0 * e[c]);
      } else {
#pragma unroll
        for (int c = 0; c < 3; ++c) tr[h][c] = (T)((2 * m * d[c] + l * trd) - (2 * mu0 * e[c] + lam0 * tre));
#pragma unroll
        for (int c = 3; c < 6; ++c) tr[h][c] = (T)(2 * m * d[c] - 2 * mu0 * e[c]);
      }
    }
#pragma unroll
    for (int c = 0; c < 6; ++c) lines[c * PL + pz] = mk<C>(tr[0][c], tr[1][c]);
  }
  __syncthreads();
  warp_fft<NZ, -1, 2>(lw, PL, tw, lane);
  for (int cc = 0; cc < 2; ++cc) {
    const int c = 2 * warp + cc;
    const C* ln = lines + c * PL;
    C* ra = spec + c * plane + l0 * ld;
    for (int k = lane; k < NZH; k += 32) {
      const C z = ln[pidx<C>(k)];
      const C w = ln[pidx<C>(k == 0 ? 0 : NZ - k)];
      ra[k] = mk<C>(T(0.5) * (z.x + w.x), T(0.5) * (z.y - w.y));
      ra[ld + k] = mk<C>(T(0.5) * (z.y + w.y), T(-0.5) * (z.x - w.x));
    }
  }
  if (!IN_SPEC) return;
  ls3d_decide<FINAL>(R, S, r, item, d2, n2, partials, rep_counter, ctl, cond, use_cond, guard_cap, red, s_last);
}

template <typename T, bool IN_SPEC, bool FINAL, int LAW = 0>
__device__ __forceinline__ void ls3d_zline_fast_entry(const Ls3dRep* __restrict__ reps, Ls3dState* st,
                                                      const int* __restrict__ map, const int* __restrict__ loc,
                                                      double* partials, unsigned int* rep_counter, Ls3dCtl* ctl,
                                                      cudaGraphConditionalHandle cond, int use_cond, int guard_cap) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ double red[32];
  __shared__ int s_last;
  __shared__ __align__(8) uint64_t bar;
  const int item = blockIdx.x;
  const int r = map[item];
  const Ls3dRep& R = reps[r];
  Ls3dState& S = st[r];
  if (IN_SPEC && use_cond && item == 0 && threadIdx.x == 0) {
    const unsigned int b = atomicAdd(&ctl->bodies, 1u) + 1u;
    if (ctl->n_active == 0 || b > (unsigned int)guard_cap || *(volatile int*)&ctl->error != 0) {
      ctl->any = 0;
      cudaGraphSetConditional(cond, 0u);
    }
  }
  if (S.done != 0) return;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    fence_mbar_init();
  }
  __syncthreads();
  const long long l0 = 2LL * loc[item];
#define MGK_Z3_CASE(n) case n: ls3_zline_body<T, IN_SPEC, FINAL, n, LAW>(R, S, item, r, l0, partials, rep_counter, ctl, cond, use_cond, guard_cap, smem_raw, &bar, red, &s_last); break;
  switch (R.nz) {
    MGK_Z3_CASE(64) MGK_Z3_CASE(96) MGK_Z3_CASE(128)
    default: break;
  }
#undef MGK_Z3_CASE
}

// FP32 phase kernel with a register target of 8 resident CTAs per SM, and
// the FP64 kernel with one of 5 (both measured faster at 128^3 than the
// compiler's own choice, despite some spilled registers)
template <typename T, bool IN_SPEC, bool FINAL>
__global__ void __launch_bounds__(96, 8) ls3d_zline_fast_kernel(const Ls3dRep* __restrict__ reps, Ls3dState* st,
                                                            const int* __restrict__ map, const int* __restrict__ loc,
                                                            double* partials, unsigned int* rep_counter, Ls3dCtl* ctl,
                                                            cudaGraphConditionalHandle cond, int use_cond,
                                                            int guard_cap) {
  ls3d_zline_fast_entry<T, IN_SPEC, FINAL>(reps, st, map, loc, partials, rep_counter, ctl, cond, use_cond, guard_cap);
}
template <bool IN_SPEC, bool FINAL, int LAW = 0>  // LAW 1: the secant law, 3: the Landau law
__global__ void __launch_bounds__(96, 5) ls3d_zline_fast64_kernel(const Ls3dRep* __restrict__ reps, Ls3dState* st,
                                                                const int* __restrict__ map, const int* __restrict__ loc,
                                                                double* partials, unsigned int* rep_counter,
                                                                Ls3dCtl* ctl, cudaGraphConditionalHandle cond,
                                                                int use_cond, int guard_cap) {
  ls3d_zline_fast_entry<double, IN_SPEC, FINAL, LAW>(reps, st, map, loc, partials, rep_counter, ctl, cond,
                                                     use_cond, guard_cap);
}

template <typename T, int AXIS, int SIGN, int NL, int NC>
__device__ __forceinline__ void ls3_axis_body(const Ls3dRep& R, const Ls3dState& S, int o, int k0, int c0,
                                              unsigned char* smem) {
  using C = C_t<T>;
  constexpr int PL = padded_len<C>(NL);
  constexpr int TC = kL3Tile;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nx = R.nx, ny = R.ny, nz = R.nz, nzh = R.nzh, ld = R.ld;
  const int tcw = min(TC, nzh - k0);
  const long long plane = (long long)nx * ny * ld;
  const long long jstride = AXIS == 1 ? ld : (long long)ny * ld;
  const long long obase = AXIS == 1 ? (long long)o * ny * ld : (long long)o * ld;
  C* lines = reinterpret_cast<C*>(smem);  // line (c * TC + t), c relative to c0
  C* spec = L3F<T>::spec(R) + c0 * plane;
  constexpr int TOT = NC * NL * TC;
  for (int e = threadIdx.x; e < TOT; e += NC * 32) {
    const int c = e / (NL * TC);
    const int rem = e - c * NL * TC;
    const int j = rem / TC, t = rem - j * TC;
    if (t < tcw) cp_async_elem(&lines[(c * TC + t) * PL + pidx<C>(j)], &spec[c * plane + obase + j * jstride + k0 + t]);
  }
  cp_async_wait_all();
  __syncthreads();
  const C* tw = reinterpret_cast<const C*>((AXIS == 1 ? L3F<T>::fy(R) : L3F<T>::fx(R)).tw);
  C* l0 = lines + warp * TC * PL;
  warp_fft<NL, AXIS == 1 ? SIGN : -1, 2>(l0, PL, tw, lane);
  warp_fft<NL, AXIS == 1 ? SIGN : -1, 2>(l0 + 2 * PL, PL, tw, lane);
  if constexpr (AXIS == 0) {
    // Gamma0 in the precision of the pass: FP64 iterations in double, the
    // FP32 phase of a mixed plan in float (its errors are those of its FP32
    // fields; the FP64 phase that follows removes both)
    __syncthreads();
    const T scale = T(1.0 / (double)R.N);
    const T inv2mu0 = (T)S.inv2mu0, Bc = (T)S.Bc;
    const int ky = o;
    const T uy = (T)fftfreq3(ky, ny) / (T)ny;
    const bool nqy = (ny & 1) == 0 && 2 * ky == ny;
    for (int e = threadIdx.x; e < tcw * NL; e += NC * 32) {
      const int t = e / NL, kx = e - t * NL;
      const int kz = k0 + t;
      const int pk = pidx<C>(kx);
      C tv[6], ev[6];
#pragma unroll
      for (int c = 0; c < 6; ++c) tv[c] = lines[(c * TC + t) * PL + pk];
      if (kx == 0 && ky == 0 && kz == 0) {
        for (int c = 0; c < 6; ++c) lines[(c * TC + t) * PL + pk] = mk<C>(T(0), T(0));
        continue;
      }
      const T ux = (T)fftfreq3(kx, nx) / (T)nx, uz = (T)fftfreq3(kz, nz) / (T)nz;
      const T inv = T(1) / sqrt(ux * ux + uy * uy + uz * uz);
      const T n0 = ux * inv, n1 = uy * inv, n2 = uz * inv;
      gamma3d_apply_t<T>(tv, n0, n1, n2, inv2mu0, Bc, ev);
      const bool nqx = (nx & 1) == 0 && 2 * kx == nx, nqz = (nz & 1) == 0 && 2 * kz == nz;
      if (nqx || nqy || nqz) {
        C fv[6];
        gamma3d_apply_t<T>(tv, nqx ? -n0 : n0, nqy ? -n1 : n1, nqz ? -n2 : n2, inv2mu0, Bc, fv);
#pragma unroll
        for (int c = 0; c < 6; ++c) ev[c] = mk<C>(T(0.5) * (ev[c].x + fv[c].x), T(0.5) * (ev[c].y + fv[c].y));
      }
#pragma unroll
      for (int c = 0; c < 6; ++c) lines[(c * TC + t) * PL + pk] = mk<C>(ev[c].x * scale, ev[c].y * scale);
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
    if (t < tcw) spec[c * plane + obase + j * jstride + k0 + t] = lines[(c * TC + t) * PL + pidx<C>(j)];
  }
}

// components per CTA of the axis kernels: the x pass applies Gamma0 across
// all 6 components; the FP64 y passes transform 3 components per CTA (two
// CTAs per tile: 5 resident CTAs of 3 warps per SM instead of 2 of 6 at the
// registers an FP64 line pair needs).  FP32 y passes keep 6 per CTA (measured
// faster at 128^3).  Second value: resident-CTA target for the allocator
// (the FP32 x pass: 3, at most 96 registers).
__host__ __device__ constexpr int ls3_axis_nc(int axis, int tsz) { return axis == 0 || tsz == 4 ? 6 : 3; }
__host__ __device__ constexpr int ls3_axis_minb(int axis, int tsz) {
  return ls3_axis_nc(axis, tsz) == 3 ? 5 : (axis == 0 && tsz == 4 ? 3 : 2);
}

// grid = items * (6 / NC), the component group fastest
template <typename T, int AXIS, int SIGN>
__global__ void __launch_bounds__(ls3_axis_nc(AXIS, sizeof(T)) * 32, ls3_axis_minb(AXIS, sizeof(T)))
    ls3d_axis_fast_kernel(const Ls3dRep* __restrict__ reps, const Ls3dState* __restrict__ st,
                          const int* __restrict__ map, const int* __restrict__ loc) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  constexpr int NC = ls3_axis_nc(AXIS, sizeof(T));
  const int item = blockIdx.x / (6 / NC);
  const int c0 = (blockIdx.x % (6 / NC)) * NC;
  const int r = map[item];
  const Ls3dRep& R = reps[r];
  const Ls3dState& S = st[r];
  if (S.done != 0) return;
  const int ntile = (R.nzh + kL3Tile - 1) / kL3Tile;
  const int o = loc[item] / ntile;
  const int k0 = (loc[item] - o * ntile) * kL3Tile;
  const int nl = AXIS == 1 ? R.ny : R.nx;
#define MGK_A3_CASE(n) case n: ls3_axis_body<T, AXIS, SIGN, n, NC>(R, S, o, k0, c0, smem_raw); break;
  switch (nl) {
    MGK_A3_CASE(64) MGK_A3_CASE(96) MGK_A3_CASE(128)
    default: break;
  }
#undef MGK_A3_CASE
}

// Mixed plans, between the phases: FP64 field from the FP32 one; grid (G, nsel)
__global__ void ls3d_promote_kernel(const Ls3dRep* reps, const int* sel) {
  const int r = sel[blockIdx.y];
  const Ls3dRep& R = reps[r];
  const long long n6 = 6 * R.N;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n6; i += (long long)gridDim.x * blockDim.x)
    R.eps[i] = (double)R.eps32[i];
}

// replicas that finished phase 1 re-enter for phase 2; resets the control block
__global__ void ls3d_phase2_kernel(Ls3dState* st, const int* sel, int nsel, Ls3dCtl* ctl) {
  if (threadIdx.x != 0) return;
  unsigned int n = 0;
  for (int q = 0; q < nsel; ++q) {
    Ls3dState& S = st[sel[q]];
    if (S.done == 1) { S.done = 0; S.phase_iter = 0; ++n; }
  }
  ctl->n_active = n;
  ctl->decided = 0;
  ctl->still = 0;
  ctl->bodies = 0;
  ctl->any = n > 0;
}

// outputs (nx,ny,nz,3,3) and partial sums for the means; grid (G, nsel)
template <int LAW = 0>  // 1: the secant law, 3: the Landau law
__global__ void ls3d_output_kernel(const Ls3dRep* reps, const Ls3dState* st, const int* sel, double* partials) {
  __shared__ double red[32];
  const int r = sel[blockIdx.y];
  const Ls3dRep& R = reps[r];
  const Ls3dState& S = st[r];
  const long long N = R.N;
  double s[18];
  for (int q = 0; q < 18; ++q) s[q] = 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N;
       i += (long long)gridDim.x * blockDim.x) {
    double e[9], p[9];
    const double sxx = R.eps[i], syy = R.eps[N + i], szz = R.eps[2 * N + i];
    const double syz = R.eps[3 * N + i], sxz = R.eps[4 * N + i], sxy = R.eps[5 * N + i];
    e[0] = sxx; e[4] = syy; e[8] = szz;
    e[1] = S.abar[0] == 0 ? sxy : sxy + S.abar[0];
    e[3] = S.abar[0] == 0 ? sxy : sxy - S.abar[0];
    e[2] = S.abar[1] == 0 ? sxz : sxz + S.abar[1];
    e[6] = S.abar[1] == 0 ? sxz : sxz - S.abar[1];
    e[5] = S.abar[2] == 0 ? syz : syz + S.abar[2];
    e[7] = S.abar[2] == 0 ? syz : syz - S.abar[2];
    if (R.epf) {
      for (int q = 0; q < 9; ++q) p[q] = R.epf[q * N + i];
    } else {
      p[0] = R.ep[i]; p[4] = R.ep[N + i]; p[8] = R.ep[2 * N + i];
      p[5] = p[7] = R.ep[3 * N + i];
      p[2] = p[6] = R.ep[4 * N + i];
      p[1] = p[3] = R.ep[5 * N + i];
    }
    double mu = R.mu[i];
    const double lam = R.lam[i];
    double d[9];
    for (int q = 0; q < 9; ++q) d[q] = e[q] - p[q];
    if constexpr (LAW == 1)
      mu = secant_mu3(mu, d[0], d[4], d[8], 0.5 * (d[5] + d[7]), 0.5 * (d[2] + d[6]), 0.5 * (d[1] + d[3]),
                      R.law_a, R.law_b);
    const double tr = d[0] + d[4] + d[8];
    double sg[9];
    if constexpr (LAW == 3) {
      // symmetric strains (the Landau solver takes symmetric tensors)
      const double a6[6] = {d[0], d[4], d[8], d[5], d[2], d[1]};
      double s6[6];
      landau_sigma3(mu, lam, a6, R.lp, s6);
      sg[0] = s6[0]; sg[4] = s6[1]; sg[8] = s6[2];
      sg[5] = sg[7] = s6[3];
      sg[2] = sg[6] = s6[4];
      sg[1] = sg[3] = s6[5];
    } else {
      for (int q = 0; q < 9; ++q) sg[q] = 2 * mu * d[q] + ((q % 4) == 0 ? lam * tr : 0.0);
    }
    for (int q = 0; q < 9; ++q) {
      if (R.out_eps) R.out_eps[9 * i + q] = e[q];
      if (R.out_sig) R.out_sig[9 * i + q] = sg[q];
      s[q] += e[q];
      s[9 + q] += sg[q];
    }
  }
  for (int q = 0; q < 18; ++q) {
    double t = block_sum(s[q], red);
    if (threadIdx.x == 0) partials[((size_t)blockIdx.y * gridDim.x + blockIdx.x) * 18 + q] = t;
  }
}

}  // namespace mgk

// ================================================================== plan ===
using namespace mgk;

namespace {
constexpr int kT3 = 256;
constexpr int kG3 = 256;
int g3(long long N) {
  long long b = (N + kT3 - 1) / kT3;
  return (int)std::max(1LL, std::min((long long)kG3, b));
}
int tc3(int n) {
  int tc = 8;
  while (tc > 1 && 2 * 6 * (size_t)tc * n * sizeof(double2) > 64 * 1024) tc >>= 1;
  return tc;
}
}  // namespace

struct mgk_ls3d_plan {
  int nrep = 0;
  long long maxN = 0;
  size_t zl_smem = 0, ax_smem = 0;
  int fast = 0;  // warp-line kernels (every side 64, 96 or 128)
  int prec = MGK_FP64;
  size_t zl_smem32 = 0, ax_smem32 = 0;
  std::vector<Ls3dRep> reps;
  std::vector<char> has_material;
  std::vector<void*> allocations;
  Ls3dRep* h_reps = nullptr;
  int* h_maps = nullptr;
  Ls3dCtl* h_ctl = nullptr;
  Ls3dState* h_state = nullptr;
  cudaEvent_t staged = nullptr;
  bool staged_pending = false;
  Ls3dRep* d_reps = nullptr;
  Ls3dState* d_st = nullptr;
  Ls3dCtl* d_ctl = nullptr;
  int* d_maps = nullptr;
  unsigned int* d_repctr = nullptr;
  double* d_part = nullptr;
  double* d_mat_part = nullptr;
  int tot_zl = 0, tot_y = 0, tot_x = 0;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int graph_mode = -1, graph_cap = 0;
  int nsel = 0, s_zl = 0, s_y = 0, s_x = 0;
  int law = 0;  // 1: secant degradation law (mgk_ls3d_set_secant)
};

static int a3(mgk_ls3d_t p, void** ptr, size_t bytes) {
  if (cudaMalloc(ptr, bytes) != cudaSuccess) {
    cudaGetLastError();
    set_error("mgk_ls3d: cudaMalloc of %zu bytes failed", bytes);
    return MGK_OOM;
  }
  p->allocations.push_back(*ptr);
  return MGK_OK;
}

// Precision form (warp-line plans only): MGK_MIXED runs FP32 iterations
// (FP32 fields, spectra and Gamma0) until the update norm is below
// max(tol, 2e-6), then FP64 iterations from that field to tol.
extern "C" int mgk_ls3d_set_precision(mgk_ls3d_t p, int precision) {
  MGK_REQUIRE(p, "mgk_ls3d_set_precision: null plan");
  MGK_REQUIRE(precision == MGK_FP64 || precision == MGK_MIXED, "mgk_ls3d_set_precision: bad precision");
  MGK_REQUIRE(precision == MGK_FP64 || p->fast,
              "mgk_ls3d_set_precision: the mixed form needs every side in {64, 96, 128}");
  if (precision == MGK_MIXED && !p->reps[0].mu32) {
    for (int r = 0; r < p->nrep; ++r) {
      Ls3dRep& R = p->reps[r];
      void* f = nullptr;
      int st = a3(p, &f, sizeof(float) * R.N * 14);
      if (st) return st;
      float* fl = reinterpret_cast<float*>(f);
      R.mu32 = fl; R.lam32 = fl + R.N; R.eps32 = fl + 2 * R.N; R.ep32 = fl + 8 * R.N;
      R.fx32 = R.fx; R.fy32 = R.fy; R.fz32 = R.fz;
      R.fx32.tw = twiddles(R.nx, 1); R.fy32.tw = twiddles(R.ny, 1); R.fz32.tw = twiddles(R.nz, 1);
      if (!R.fx32.tw || !R.fy32.tw || !R.fz32.tw) return MGK_OOM;
      p->has_material[r] = 0;  // the FP32 copies come with the next set_material
    }
    MGK_CUDA(cudaMemcpy(p->d_reps, p->reps.data(), sizeof(Ls3dRep) * p->nrep, cudaMemcpyHostToDevice));
  }
  if (precision != p->prec) p->graph_mode = -1;
  p->prec = precision;
  return MGK_OK;
}

extern "C" int mgk_ls3d_destroy(mgk_ls3d_t p) {
  if (!p) return MGK_OK;
  if (p->exec) cudaGraphExecDestroy(p->exec);
  if (p->graph) cudaGraphDestroy(p->graph);
  if (p->staged) cudaEventDestroy(p->staged);
  for (void* a : p->allocations) cudaFree(a);
  if (p->h_reps) cudaFreeHost(p->h_reps);
  if (p->h_maps) cudaFreeHost(p->h_maps);
  if (p->h_ctl) cudaFreeHost(p->h_ctl);
  if (p->h_state) cudaFreeHost(p->h_state);
  delete p;
  return MGK_OK;
}

extern "C" int mgk_ls3d_create_batch(int nrep, const int* nxs, const int* nys, const int* nzs, mgk_ls3d_t* out) {
  MGK_REQUIRE(out, "mgk_ls3d_create: null output handle");
  *out = nullptr;
  MGK_REQUIRE(nrep >= 1 && nrep <= 4096 && nxs && nys && nzs, "mgk_ls3d_create: bad replica count");
  for (int r = 0; r < nrep; ++r) {
    FftLen f;
    MGK_REQUIRE(fft_schedule(nxs[r], &f) && fft_schedule(nys[r], &f) && fft_schedule(nzs[r], &f),
                "mgk_ls3d_create: grid %dx%dx%d unsupported (each side 2^a 3^b up to 4096)", nxs[r], nys[r],
                nzs[r]);
    MGK_REQUIRE(((long long)nxs[r] * nys[r]) % 2 == 0 /* z-lines are transformed in pairs */ && 2 * 6 * (size_t)nzs[r] * sizeof(double2) <= 220 * 1024 &&
                    2 * 6 * (size_t)tc3(std::max(nxs[r], nys[r])) * std::max(nxs[r], nys[r]) * sizeof(double2) <=
                        220 * 1024,
                "mgk_ls3d_create: grid too large for the shared-memory FFT");
  }
  mgk_ls3d_t p = new mgk_ls3d_plan();
  auto fail = [&](int s) { mgk_ls3d_destroy(p); return s; };
  p->nrep = nrep;
  p->reps.resize(nrep);
  p->has_material.assign(nrep, 0);
  {
    bool fast = true;
    for (int r = 0; r < nrep; ++r) fast = fast && ls3_fast_len(nxs[r]) && ls3_fast_len(nys[r]) && ls3_fast_len(nzs[r]);
    const char* env = getenv("MGK_FAST");
    p->fast = fast && !(env && env[0] == '0');
  }
  for (int r = 0; r < nrep; ++r) {
    Ls3dRep& R = p->reps[r];
    memset(&R, 0, sizeof(R));
    R.nx = nxs[r]; R.ny = nys[r]; R.nz = nzs[r];
    R.nzh = R.nz / 2 + 1;
    R.ld = R.nzh;
    R.N = (long long)R.nx * R.ny * R.nz;
    R.tc = p->fast ? kL3Tile : tc3(std::max(R.nx, R.ny));
    const int ntile = (R.nzh + R.tc - 1) / R.tc;
    R.zl_items = R.nx * R.ny / 2;
    R.y_items = R.nx * ntile;
    R.x_items = R.ny * ntile;
    fft_schedule(R.nx, &R.fx); fft_schedule(R.ny, &R.fy); fft_schedule(R.nz, &R.fz);
    R.fx.tw = twiddles(R.nx, MGK_FP64); R.fy.tw = twiddles(R.ny, MGK_FP64); R.fz.tw = twiddles(R.nz, MGK_FP64);
    if (!R.fx.tw || !R.fy.tw || !R.fz.tw) return fail(MGK_OOM);
    if (p->fast) {
      p->zl_smem = std::max(p->zl_smem, (size_t)ls3_zl_smem(R.nz, 16));
      p->ax_smem = std::max(p->ax_smem, (size_t)ls3_ax_smem(std::max(R.nx, R.ny), 16));
      p->zl_smem32 = std::max(p->zl_smem32, (size_t)ls3_zl_smem(R.nz, 8));
      p->ax_smem32 = std::max(p->ax_smem32, (size_t)ls3_ax_smem(std::max(R.nx, R.ny), 8));
    } else {
      p->zl_smem = std::max(p->zl_smem, 2 * 6 * (size_t)R.nz * sizeof(double2));
      p->ax_smem = std::max(p->ax_smem, 2 * 6 * (size_t)R.tc * std::max(R.nx, R.ny) * sizeof(double2));
    }
    p->maxN = std::max(p->maxN, R.N);
    p->tot_zl += R.zl_items; p->tot_y += R.y_items; p->tot_x += R.x_items;
    void* f = nullptr;
    int st = a3(p, &f, sizeof(double) * R.N * 23);
    if (st) return fail(st);
    double* d = reinterpret_cast<double*>(f);
    R.mu = d; R.lam = d + R.N; R.eps = d + 2 * R.N; R.ep = d + 8 * R.N; R.epf = nullptr;
    void* sp = nullptr;
    st = a3(p, &sp, 6 * (size_t)R.nx * R.ny * R.ld * sizeof(double2));
    if (st) return fail(st);
    R.spec = reinterpret_cast<double2*>(sp);
  }
  int st;
  if (p->fast &&
      (raise_smem((const void*)ls3d_zline_fast64_kernel<true, true>, (int)p->zl_smem) ||
       raise_smem((const void*)ls3d_zline_fast64_kernel<false, true>, (int)p->zl_smem) ||
       raise_smem((const void*)ls3d_zline_fast64_kernel<true, true, 1>, (int)p->zl_smem) ||
       raise_smem((const void*)ls3d_zline_fast64_kernel<false, true, 1>, (int)p->zl_smem) ||
       raise_smem((const void*)ls3d_zline_fast64_kernel<true, true, 3>, (int)p->zl_smem) ||
       raise_smem((const void*)ls3d_zline_fast64_kernel<false, true, 3>, (int)p->zl_smem) ||
       raise_smem((const void*)ls3d_axis_fast_kernel<double, 1, -1>, (int)p->ax_smem) ||
       raise_smem((const void*)ls3d_axis_fast_kernel<double, 1, 1>, (int)p->ax_smem) ||
       raise_smem((const void*)ls3d_axis_fast_kernel<double, 0, 0>, (int)p->ax_smem) ||
       raise_smem((const void*)ls3d_zline_fast_kernel<float, true, false>, (int)p->zl_smem32) ||
       raise_smem((const void*)ls3d_zline_fast_kernel<float, false, false>, (int)p->zl_smem32) ||
       raise_smem((const void*)ls3d_axis_fast_kernel<float, 1, -1>, (int)p->ax_smem32) ||
       raise_smem((const void*)ls3d_axis_fast_kernel<float, 1, 1>, (int)p->ax_smem32) ||
       raise_smem((const void*)ls3d_axis_fast_kernel<float, 0, 0>, (int)p->ax_smem32))) {
    set_error("mgk_ls3d_create: cudaFuncSetAttribute failed");
    return fail(MGK_CUDA_ERROR);
  }
  if (!p->fast && (raise_smem((const void*)ls3d_zline_kernel<true>, (int)p->zl_smem) ||
      raise_smem((const void*)ls3d_zline_kernel<false>, (int)p->zl_smem) ||
      raise_smem((const void*)ls3d_axis_kernel<1, -1>, (int)p->ax_smem) ||
      raise_smem((const void*)ls3d_axis_kernel<1, 1>, (int)p->ax_smem) ||
      raise_smem((const void*)ls3d_axis_kernel<0, 0>, (int)p->ax_smem))) {
    set_error("mgk_ls3d_create: cudaFuncSetAttribute failed");
    return fail(MGK_CUDA_ERROR);
  }
  const int G = g3(p->maxN);
  const size_t part = std::max((size_t)2 * p->tot_zl, (size_t)nrep * G * 18);
  void* v = nullptr;
  if ((st = a3(p, &v, sizeof(double) * part))) return fail(st);
  p->d_part = reinterpret_cast<double*>(v);
  if ((st = a3(p, &v, sizeof(double) * 2 * kG3))) return fail(st);
  p->d_mat_part = reinterpret_cast<double*>(v);
  if ((st = a3(p, &v, sizeof(Ls3dRep) * nrep))) return fail(st);
  p->d_reps = reinterpret_cast<Ls3dRep*>(v);
  if ((st = a3(p, &v, sizeof(Ls3dState) * nrep))) return fail(st);
  p->d_st = reinterpret_cast<Ls3dState*>(v);
  if ((st = a3(p, &v, sizeof(Ls3dCtl)))) return fail(st);
  p->d_ctl = reinterpret_cast<Ls3dCtl*>(v);
  const size_t nm = 2 * (size_t)(p->tot_zl + p->tot_y + p->tot_x) + nrep;
  if ((st = a3(p, &v, sizeof(int) * nm))) return fail(st);
  p->d_maps = reinterpret_cast<int*>(v);
  if ((st = a3(p, &v, sizeof(unsigned int) * nrep))) return fail(st);
  p->d_repctr = reinterpret_cast<unsigned int*>(v);
  if (cudaMemset(p->d_repctr, 0, sizeof(unsigned int) * nrep) || cudaMemset(p->d_st, 0, sizeof(Ls3dState) * nrep) ||
      cudaMemset(p->d_ctl, 0, sizeof(Ls3dCtl)))
    return fail(MGK_CUDA_ERROR);
  if (cudaMallocHost(&p->h_reps, sizeof(Ls3dRep) * nrep) || cudaMallocHost(&p->h_maps, sizeof(int) * nm) ||
      cudaMallocHost(&p->h_ctl, sizeof(Ls3dCtl)) || cudaMallocHost(&p->h_state, sizeof(Ls3dState) * nrep))
    return fail(MGK_OOM);
  if (cudaEventCreateWithFlags(&p->staged, cudaEventDisableTiming)) return fail(MGK_CUDA_ERROR);
  memcpy(p->h_reps, p->reps.data(), sizeof(Ls3dRep) * nrep);
  if (cudaMemcpy(p->d_reps, p->h_reps, sizeof(Ls3dRep) * nrep, cudaMemcpyHostToDevice)) return fail(MGK_CUDA_ERROR);
  *out = p;
  return MGK_OK;
}

extern "C" int mgk_ls3d_create(int nx, int ny, int nz, mgk_ls3d_t* out) {
  return mgk_ls3d_create_batch(1, &nx, &ny, &nz, out);
}

static int wait3(mgk_ls3d_t p) {
  if (p->staged_pending) {
    MGK_CUDA(cudaEventSynchronize(p->staged));
    p->staged_pending = false;
  }
  return MGK_OK;
}

static int set3(mgk_ls3d_t p, int rep, const double* E, const double* nu, const double* epsp, int set_moduli,
                cudaStream_t s) {
  Ls3dRep& R = p->reps[rep];
  const bool want = epsp != nullptr;
  if (want != (R.epf != nullptr)) {
    R.epf = want ? R.mu + 14 * R.N : nullptr;
    int st = wait3(p);
    if (st) return st;
    p->h_reps[rep] = R;
    MGK_CUDA(cudaMemcpyAsync(&p->d_reps[rep], &p->h_reps[rep], sizeof(Ls3dRep), cudaMemcpyHostToDevice, s));
    MGK_CUDA(cudaEventRecord(p->staged, s));
    p->staged_pending = true;
  }
  const int G = g3(R.N);
  ls3d_material_kernel<<<G, kT3, 0, s>>>(p->d_reps, rep, E, nu, epsp, set_moduli, p->d_mat_part);
  MGK_CUDA(cudaGetLastError());
  if (set_moduli) {
    ls3d_medium_kernel<<<1, kT3, 0, s>>>(p->d_reps, p->d_st, rep, p->d_mat_part, G, set_moduli == 2);
    MGK_CUDA(cudaGetLastError());
  }
  return MGK_OK;
}

extern "C" int mgk_ls3d_set_material_rep(mgk_ls3d_t p, int rep, const double* E, const double* nu,
                                         const double* epsp, mgk_stream_t stream) {
  MGK_REQUIRE(p && E && nu && rep >= 0 && rep < p->nrep, "mgk_ls3d_set_material: bad argument");
  int st = set3(p, rep, E, nu, epsp, 1, (cudaStream_t)stream);
  if (st == MGK_OK) p->has_material[rep] = 1;
  return st;
}

extern "C" int mgk_ls3d_set_lame_rep(mgk_ls3d_t p, int rep, const double* lam, const double* mu,
                                     const double* epsp, mgk_stream_t stream) {
  MGK_REQUIRE(p && lam && mu && rep >= 0 && rep < p->nrep, "mgk_ls3d_set_lame: bad argument");
  int st = set3(p, rep, lam, mu, epsp, 2, (cudaStream_t)stream);
  if (st == MGK_OK) p->has_material[rep] = 1;
  return st;
}

// every replica to the secant law (d > 0) or back to the linear law; cached
// loop graphs hold the previous law's z-line kernel and are dropped
extern "C" int mgk_ls3d_set_secant(mgk_ls3d_t p, double d, double k) {
  MGK_REQUIRE(p, "mgk_ls3d_set_secant: null plan");
  MGK_REQUIRE(d >= 0.0 && d <= 1.0 && k >= 0.0 && isfinite(k), "mgk_ls3d_set_secant: need 0 <= d <= 1, k >= 0");
  MGK_REQUIRE(d == 0.0 || p->prec == MGK_FP64, "mgk_ls3d_set_secant: the secant law runs in FP64 plans only");
  const int law = d != 0.0 ? 1 : 0;
  for (auto& R : p->reps) { R.law = law; R.law_a = d; R.law_b = k; }
  if (law != p->law) {
    if (p->graph_mode == 1) p->graph_mode = -1;
    p->law = law;
  }
  return MGK_OK;
}

// every replica to the Landau law (spectral_solver_landau_3d); cached loop
// graphs hold the previous law's z-line kernel and are dropped
extern "C" int mgk_ls3d_set_landau(mgk_ls3d_t p, const double* v, int capping, double e_cap, double tangent_ratio,
                                   double smooth_power) {
  MGK_REQUIRE(p && v, "mgk_ls3d_set_landau: null argument");
  MGK_REQUIRE(p->prec == MGK_FP64, "mgk_ls3d_set_landau: the Landau law runs in FP64 plans only");
  MGK_REQUIRE(capping >= 0 && capping <= 2, "mgk_ls3d_set_landau: capping must be 0, 1 or 2");
  MGK_REQUIRE(capping == 0 || (e_cap > 0.0 && (capping != 2 || smooth_power > 0.0)),
              "mgk_ls3d_set_landau: need e_cap > 0 (and smooth_power > 0 for smooth capping)");
  for (int q = 0; q < 7; ++q) MGK_REQUIRE(isfinite(v[q]), "mgk_ls3d_set_landau: non-finite coefficient");
  for (auto& R : p->reps) {
    R.law = 3;
    for (int q = 0; q < 7; ++q) R.lp[q] = v[q];
    R.lp[7] = capping;
    R.lp[8] = e_cap;
    R.lp[9] = tangent_ratio;
    R.lp[10] = smooth_power;
  }
  if (p->law != 3) {
    if (p->graph_mode == 1) p->graph_mode = -1;
    p->law = 3;
  }
  return MGK_OK;
}

extern "C" int mgk_ls3d_set_eigenstrain_rep(mgk_ls3d_t p, int rep, const double* epsp, mgk_stream_t stream) {
  MGK_REQUIRE(p && rep >= 0 && rep < p->nrep && p->has_material[rep], "mgk_ls3d_set_eigenstrain: no material");
  return set3(p, rep, nullptr, nullptr, epsp, 0, (cudaStream_t)stream);
}

struct Loop3 {
  const Ls3dRep* reps;
  Ls3dState* st;
  const int *zm, *zl, *ym, *yl, *xm, *xl;
  double* part;
  unsigned int* ctr;
  Ls3dCtl* ctl;
  int nzl, ny, nx;
  size_t zs, as;
  int fast;
  // mixed plans: FP32 phase shared memory, the selection and the
  // per-voxel grid of the promote kernel
  size_t zs32, as32;
  const int* sel;
  int nsel, G;
  int law;
};

// kernels of one iteration: `f32` selects the FP32 phase of a mixed plan
// (warp-line kernels only; its decisions end phase 1, not the solve)
static void* zline_fn(int fast, bool in_spec, bool f32 = false, int law = 0) {
  if (fast && !f32 && law == 1)
    return in_spec ? (void*)ls3d_zline_fast64_kernel<true, true, 1> : (void*)ls3d_zline_fast64_kernel<false, true, 1>;
  if (fast && !f32 && law == 3)
    return in_spec ? (void*)ls3d_zline_fast64_kernel<true, true, 3> : (void*)ls3d_zline_fast64_kernel<false, true, 3>;
  if (fast && f32)
    return in_spec ? (void*)ls3d_zline_fast_kernel<float, true, false> : (void*)ls3d_zline_fast_kernel<float, false, false>;
  if (fast)
    return in_spec ? (void*)ls3d_zline_fast64_kernel<true, true> : (void*)ls3d_zline_fast64_kernel<false, true>;
  return in_spec ? (void*)ls3d_zline_kernel<true> : (void*)ls3d_zline_kernel<false>;
}
template <int AXIS, int SIGN> static void* axis_fn(int fast, bool f32 = false) {
  if (fast && f32) return (void*)ls3d_axis_fast_kernel<float, AXIS, SIGN>;
  return fast ? (void*)ls3d_axis_fast_kernel<double, AXIS, SIGN> : (void*)ls3d_axis_kernel<AXIS, SIGN>;
}

static int body3(const Loop3& a, cudaStream_t s, bool f32 = false) {
  const dim3 ab(a.fast ? 192 : kT3), zb(a.fast ? 96 : kT3);
  const size_t as = f32 ? a.as32 : a.as, zs = f32 ? a.zs32 : a.zs;
  const bool ysplit = a.fast && ls3_axis_nc(1, f32 ? 4 : 8) == 3;  // FP64 y passes: 3 components per CTA
  const size_t asy = ysplit ? as / 2 : as;
  const dim3 gy(ysplit ? 2 * a.ny : a.ny), aby(ysplit ? 96 : ab.x);
  void* ay[] = {(void*)&a.reps, (void*)&a.st, (void*)&a.ym, (void*)&a.yl};
  void* ax[] = {(void*)&a.reps, (void*)&a.st, (void*)&a.xm, (void*)&a.xl};
  cudaGraphConditionalHandle h = 0;
  int zero = 0;
  void* az[] = {(void*)&a.reps, (void*)&a.st, (void*)&a.zm, (void*)&a.zl, (void*)&a.part, (void*)&a.ctr,
                (void*)&a.ctl, &h, &zero, &zero};
  MGK_CUDA(cudaLaunchKernel(axis_fn<1, -1>(a.fast, f32), gy, aby, ay, asy, s));
  MGK_CUDA(cudaLaunchKernel(axis_fn<0, 0>(a.fast, f32), dim3(a.nx), ab, ax, as, s));
  MGK_CUDA(cudaLaunchKernel(axis_fn<1, 1>(a.fast, f32), gy, aby, ay, asy, s));
  MGK_CUDA(cudaLaunchKernel(zline_fn(a.fast, true, f32, a.law), dim3(a.nzl), zb, az, zs, s));
  return MGK_OK;
}

// one while node running iterations of the FP32 (phase 1) or FP64 kernels
static int add_while3(cudaGraph_t g, const cudaGraphNode_t* dep, Loop3& a, bool f32, int* cap,
                      cudaGraphNode_t* out) {
  cudaGraphConditionalHandle h;
  if (cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault)) return MGK_CUDA_ERROR;
  alignas(cudaGraphNodeParams) unsigned char raw[sizeof(cudaGraphNodeParams)];
  memset(raw, 0, sizeof(raw));
  cudaGraphNodeParams& cp = *reinterpret_cast<cudaGraphNodeParams*>(raw);
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = h;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  if (cudaGraphAddNode(out, g, dep, dep ? 1 : 0, &cp)) return MGK_CUDA_ERROR;
  cudaGraph_t body = cp.conditional.phGraph_out[0];
  cudaGraphNode_t prev = nullptr, node;
  auto add = [&](void* fn, dim3 grid, size_t smem, void** args, int block) {
    cudaKernelNodeParams k;
    memset(&k, 0, sizeof(k));
    k.func = fn; k.gridDim = grid; k.blockDim = dim3(block); k.sharedMemBytes = (unsigned)smem; k.kernelParams = args;
    cudaError_t e = cudaGraphAddKernelNode(&node, body, prev ? &prev : nullptr, prev ? 1 : 0, &k);
    prev = node;
    return e;
  };
  void* ay[] = {&a.reps, &a.st, &a.ym, &a.yl};
  void* ax[] = {&a.reps, &a.st, &a.xm, &a.xl};
  int use = 1;
  void* az[] = {&a.reps, &a.st, &a.zm, &a.zl, &a.part, &a.ctr, &a.ctl, &h, &use, cap};
  const int ab = a.fast ? 192 : kT3, zb = a.fast ? 96 : kT3;
  const size_t as = f32 ? a.as32 : a.as, zs = f32 ? a.zs32 : a.zs;
  const bool ysplit = a.fast && ls3_axis_nc(1, f32 ? 4 : 8) == 3;  // FP64 y passes: 3 components per CTA
  const size_t asy = ysplit ? as / 2 : as;
  const dim3 gy(ysplit ? 2 * a.ny : a.ny);
  const int aby = ysplit ? 96 : ab;
  cudaError_t e = add(axis_fn<1, -1>(a.fast, f32), gy, asy, ay, aby);
  if (!e) e = add(axis_fn<0, 0>(a.fast, f32), dim3(a.nx), as, ax, ab);
  if (!e) e = add(axis_fn<1, 1>(a.fast, f32), gy, asy, ay, aby);
  if (!e) e = add(zline_fn(a.fast, true, f32, a.law), dim3(a.nzl), zs, az, zb);
  return e ? MGK_CUDA_ERROR : MGK_OK;
}

// Loop graph: FP64 plans one while node; mixed plans [FP32 while, promote,
// phase-2 set-up, first FP64 z-line pass, FP64 while].
static int graph3(mgk_ls3d_t p, Loop3& a, int cap) {
  if (p->exec) { cudaGraphExecDestroy(p->exec); p->exec = nullptr; }
  if (p->graph) { cudaGraphDestroy(p->graph); p->graph = nullptr; }
  cudaGraph_t g;
  MGK_CUDA(cudaGraphCreate(&g, 0));
  int capv = cap;
  int rc = MGK_OK;
  cudaGraphNode_t last;
  if (p->prec == MGK_MIXED) {
    cudaGraphNode_t w1, np, n2, nz0;
    rc = add_while3(g, nullptr, a, true, &capv, &w1);
    if (rc == MGK_OK) {
      cudaKernelNodeParams k;
      memset(&k, 0, sizeof(k));
      void* ap[] = {&a.reps, (void*)&a.sel};
      k.func = (void*)ls3d_promote_kernel; k.gridDim = dim3(a.G, a.nsel); k.blockDim = dim3(kT3); k.kernelParams = ap;
      if (cudaGraphAddKernelNode(&np, g, &w1, 1, &k)) rc = MGK_CUDA_ERROR;
    }
    if (rc == MGK_OK) {
      cudaKernelNodeParams k;
      memset(&k, 0, sizeof(k));
      void* ap[] = {&a.st, (void*)&a.sel, &a.nsel, &a.ctl};
      k.func = (void*)ls3d_phase2_kernel; k.gridDim = dim3(1); k.blockDim = dim3(32); k.kernelParams = ap;
      if (cudaGraphAddKernelNode(&n2, g, &np, 1, &k)) rc = MGK_CUDA_ERROR;
    }
    if (rc == MGK_OK) {
      cudaKernelNodeParams k;
      memset(&k, 0, sizeof(k));
      cudaGraphConditionalHandle h0 = 0;
      int zero = 0;
      void* ap[] = {&a.reps, &a.st, &a.zm, &a.zl, &a.part, &a.ctr, &a.ctl, &h0, &zero, &zero};
      k.func = zline_fn(a.fast, false, false); k.gridDim = dim3(a.nzl); k.blockDim = dim3(a.fast ? 96 : kT3);
      k.sharedMemBytes = (unsigned)a.zs; k.kernelParams = ap;
      if (cudaGraphAddKernelNode(&nz0, g, &n2, 1, &k)) rc = MGK_CUDA_ERROR;
    }
    if (rc == MGK_OK) rc = add_while3(g, &nz0, a, false, &capv, &last);
  } else {
    rc = add_while3(g, nullptr, a, false, &capv, &last);
  }
  cudaGraphExec_t x = nullptr;
  if (rc == MGK_OK && cudaGraphInstantiate(&x, g, 0)) rc = MGK_CUDA_ERROR;
  if (rc) { cudaGraphDestroy(g); cudaGetLastError(); return MGK_CUDA_ERROR; }
  p->graph = g;
  p->exec = x;
  return MGK_OK;
}

extern "C" int mgk_ls3d_solve_batch(mgk_ls3d_t p, int nsel, const int* sel, const double* eps_bar,
                                    const double* const* eps_init, double* const* eps_out, double* const* sig_out,
                                    int max_iter, double tol, mgk_ls_info3* infos, mgk_stream_t stream) {
  MGK_REQUIRE(p && eps_bar && nsel >= 1 && nsel <= p->nrep, "mgk_ls3d_solve_batch: bad argument");
  MGK_REQUIRE(max_iter >= 0 && max_iter <= 1000000, "mgk_ls3d_solve: max_iter out of range");
  cudaStream_t s = (cudaStream_t)stream;
  std::vector<int> selv(nsel);
  std::vector<char> seen(p->nrep, 0);
  for (int q = 0; q < nsel; ++q) {
    const int r = sel ? sel[q] : q;
    MGK_REQUIRE(r >= 0 && r < p->nrep && !seen[r], "mgk_ls3d_solve_batch: bad or repeated replica index");
    MGK_REQUIRE(p->has_material[r], "mgk_ls3d_solve: replica %d has no material", r);
    seen[r] = 1;
    selv[q] = r;
  }
  int rc = wait3(p);
  if (rc) return rc;
  int nzl = 0, ny_ = 0, nx_ = 0;
  for (int r : selv) { nzl += p->reps[r].zl_items; ny_ += p->reps[r].y_items; nx_ += p->reps[r].x_items; }
  const bool changed = nzl != p->s_zl || ny_ != p->s_y || nx_ != p->s_x || nsel != p->nsel;
  int* zm = p->h_maps; int* zl = zm + nzl; int* ym = zl + nzl; int* yl = ym + ny_;
  int* xm = yl + ny_; int* xl = xm + nx_; int* sp = xl + nx_;
  int zi = 0, yi = 0, xi = 0;
  for (int q = 0; q < nsel; ++q) {
    const int r = selv[q];
    Ls3dRep& H = p->h_reps[r];
    H = p->reps[r];
    H.init = eps_init ? eps_init[q] : nullptr;
    H.out_eps = eps_out ? eps_out[q] : nullptr;
    H.out_sig = sig_out ? sig_out[q] : nullptr;
    for (int k = 0; k < 9; ++k) H.eb[k] = eps_bar[9 * q + k];
    H.tol = tol;
    H.max_iter = max_iter;
    H.zl_first = zi;
    for (int i = 0; i < H.zl_items; ++i) { zm[zi] = r; zl[zi] = i; ++zi; }
    for (int i = 0; i < H.y_items; ++i) { ym[yi] = r; yl[yi] = i; ++yi; }
    for (int i = 0; i < H.x_items; ++i) { xm[xi] = r; xl[xi] = i; ++xi; }
    sp[q] = r;
  }
  const int n_active = max_iter > 0 ? nsel : 0;
  *p->h_ctl = Ls3dCtl{(unsigned int)n_active, 0u, 0u, 0u, n_active > 0, 0};
  const size_t nm = 2 * (size_t)(nzl + ny_ + nx_) + nsel;
  MGK_CUDA(cudaMemcpyAsync(p->d_maps, p->h_maps, sizeof(int) * nm, cudaMemcpyHostToDevice, s));
  MGK_CUDA(cudaMemcpyAsync(p->d_reps, p->h_reps, sizeof(Ls3dRep) * p->nrep, cudaMemcpyHostToDevice, s));
  MGK_CUDA(cudaMemcpyAsync(p->d_ctl, p->h_ctl, sizeof(Ls3dCtl), cudaMemcpyHostToDevice, s));
  MGK_CUDA(cudaEventRecord(p->staged, s));
  p->staged_pending = true;
  p->s_zl = nzl; p->s_y = ny_; p->s_x = nx_; p->nsel = nsel;
  const int* d_zm = p->d_maps; const int* d_zl = d_zm + nzl; const int* d_ym = d_zl + nzl;
  const int* d_yl = d_ym + ny_; const int* d_xm = d_yl + ny_; const int* d_xl = d_xm + nx_;
  const int* d_sel = d_xl + nx_;
  const int G = g3(p->maxN);
  bool any_init = false;
  for (int q = 0; q < nsel && eps_init; ++q) any_init |= eps_init[q] != nullptr;
  if (any_init) {
    ls3d_means_kernel<<<dim3(G, nsel), kT3, 0, s>>>(p->d_reps, d_sel, p->d_part);
    ls3d_finalize_kernel<<<nsel, kT3, 0, s>>>(p->d_reps, p->d_st, d_sel, p->d_part, G, 9,
                                              (int)offsetof(Ls3dState, means), 1);
    MGK_CUDA(cudaGetLastError());
  }
  ls3d_begin_kernel<<<dim3(G, nsel), kT3, 0, s>>>(p->d_reps, p->d_st, d_sel, p->d_part);
  MGK_CUDA(cudaGetLastError());
  if (any_init) {
    ls3d_finalize_kernel<<<nsel, kT3, 0, s>>>(p->d_reps, p->d_st, d_sel, p->d_part, G, 2,
                                              (int)offsetof(Ls3dState, extra_d0), 2);
    MGK_CUDA(cudaGetLastError());
  }
  if (n_active > 0) {
    Loop3 a{p->d_reps, p->d_st, d_zm, d_zl, d_ym, d_yl, d_xm, d_xl, p->d_part, p->d_repctr, p->d_ctl,
            nzl, ny_, nx_, p->zl_smem, p->ax_smem, p->fast, p->zl_smem32, p->ax_smem32, d_sel, nsel, G, p->law};
    const bool mixed = p->prec == MGK_MIXED;
    {
      cudaGraphConditionalHandle h0 = 0;
      int zero = 0;
      void* az0[] = {(void*)&p->d_reps, (void*)&p->d_st, (void*)&d_zm, (void*)&d_zl, (void*)&p->d_part,
                     (void*)&p->d_repctr, (void*)&p->d_ctl, &h0, &zero, &zero};
      MGK_CUDA(cudaLaunchKernel(zline_fn(p->fast, false, mixed, p->law), dim3(nzl), dim3(p->fast ? 96 : kT3), az0,
                                mixed ? p->zl_smem32 : p->zl_smem, s));
    }
    const int cap = max_iter + 2 > 1000 ? max_iter + 2 : 1000;
    if (p->graph_mode == 1 && (changed || cap > p->graph_cap)) p->graph_mode = -1;
    if (p->graph_mode < 0) {
      const char* env = getenv("MGK_NO_GRAPH_WHILE");
      if (env && env[0] == '1') p->graph_mode = 0;
      else {
        p->graph_mode = graph3(p, a, cap) == MGK_OK ? 1 : 0;
        p->graph_cap = cap;
      }
    }
    if (p->graph_mode == 1) {
      MGK_CUDA(cudaGraphLaunch(p->exec, s));
    } else {
      for (int phase = mixed ? 1 : 2; phase <= 2; ++phase) {
        if (phase == 2 && mixed) {
          ls3d_promote_kernel<<<dim3(G, nsel), kT3, 0, s>>>(p->d_reps, d_sel);
          ls3d_phase2_kernel<<<1, 32, 0, s>>>(p->d_st, d_sel, nsel, p->d_ctl);
          cudaGraphConditionalHandle h0 = 0;
          int zero = 0;
          void* az1[] = {(void*)&p->d_reps, (void*)&p->d_st, (void*)&d_zm, (void*)&d_zl, (void*)&p->d_part,
                         (void*)&p->d_repctr, (void*)&p->d_ctl, &h0, &zero, &zero};
          MGK_CUDA(cudaLaunchKernel(zline_fn(p->fast, false, false, p->law), dim3(nzl), dim3(96), az1, p->zl_smem, s));
        }
        for (int it = 0; it < max_iter; ++it) {
          rc = body3(a, s, phase == 1);
          if (rc) return rc;
          Ls3dCtl hc;
          MGK_CUDA(cudaMemcpyAsync(&hc, p->d_ctl, sizeof(Ls3dCtl), cudaMemcpyDeviceToHost, s));
          MGK_CUDA(cudaStreamSynchronize(s));
          if (!hc.any) break;
        }
      }
    }
  }
  if (p->law == 1)
    ls3d_output_kernel<1><<<dim3(G, nsel), kT3, 0, s>>>(p->d_reps, p->d_st, d_sel, p->d_part);
  else if (p->law == 3)
    ls3d_output_kernel<3><<<dim3(G, nsel), kT3, 0, s>>>(p->d_reps, p->d_st, d_sel, p->d_part);
  else
    ls3d_output_kernel<0><<<dim3(G, nsel), kT3, 0, s>>>(p->d_reps, p->d_st, d_sel, p->d_part);
  MGK_CUDA(cudaGetLastError());
  ls3d_finalize_kernel<<<nsel, kT3, 0, s>>>(p->d_reps, p->d_st, d_sel, p->d_part, G, 18,
                                            (int)offsetof(Ls3dState, out_eps_mean), 0);
  MGK_CUDA(cudaGetLastError());
  if (infos) {
    MGK_CUDA(cudaMemcpyAsync(p->h_state, p->d_st, sizeof(Ls3dState) * p->nrep, cudaMemcpyDeviceToHost, s));
    Ls3dCtl hc3;
    MGK_CUDA(cudaMemcpyAsync(&hc3, p->d_ctl, sizeof(Ls3dCtl), cudaMemcpyDeviceToHost, s));
    MGK_CUDA(cudaStreamSynchronize(s));
    if (hc3.error) {
      set_error("mgk_ls3d_solve: a bulk copy wait gave up (device timeout)");
      return MGK_TIMEOUT;
    }
    int worst = MGK_OK;
    for (int q = 0; q < nsel; ++q) {
      const Ls3dState& S = p->h_state[selv[q]];
      infos[q].iterations = S.iter;
      infos[q].status = S.status;
      infos[q].final_diff = S.diff;
      for (int k = 0; k < 9; ++k) { infos[q].eps_mean[k] = S.out_eps_mean[k]; infos[q].sig_mean[k] = S.out_sig_mean[k]; }
      if (S.status == MGK_NONFINITE) worst = MGK_NONFINITE;
    }
    if (worst) { set_error("mgk_ls3d_solve: non-finite residual"); return worst; }
  }
  return MGK_OK;
}
