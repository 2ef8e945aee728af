// 2D small-strain Lippmann-Schwinger solver, batched over replicas.
//
// Restates mgkmc/linear_elastic_simulator.py:12-88 (spectral_solver_2d):
//   tau = C:(eps - eps_p) - C0:eps;  eps_new = eps_bar - IFFT(Gamma0 : FFT(tau));
//   diff = ||eps_new - eps|| / (||eps|| + 1e-20); stop when diff < tol.
// with the Green operator of mgkmc/elasticity.py:20-53 evaluated on the fly
// from the wave vector (never materialised).
//
// A plan holds `nrep` independent replicas (grids of any supported size, so a
// batch may be ragged).  A solve call selects a subset of them; every stage
// is one launch over all selected replicas.
//
// HBM layout per replica (SoA planes of N = nx*ny, C order):
//   mu, lam                 Lame fields (plane strain or plane stress lambda)
//   eps[3]                  xx, yy, symmetric xy of the current iterate
//   ep[3]                   xx, yy, symmetric xy of the eigenstrain
//   epa[2] (optional)       eps_p xy and yx when an eigenstrain is given
//   spec[3]                 half spectrum, nx rows of ld = ny/2+1 complex
// Mixed-precision plans also hold FP32 copies of mu, lam, eps and ep.  The
// antisymmetric part of eps is uniform after the first iteration (Gamma0
// returns symmetric tensors), so it is carried as one scalar.
//
// One iteration = two kernels:
//   row kernel  (one CTA per pair of x-rows): C2R along y of the previous
//               spectrum (two real rows packed as one complex line), update
//               eps = eps_bar + eps~, the diff/norm partial sums, then the
//               polarisation tau and the R2C along y of the next iteration;
//   column kernel (one CTA per tile of ky columns): complex FFT along x,
//               eps~^ = -Gamma0_sym(k) : tau^ / N, inverse FFT along x.
// The spectral field crosses HBM once per direction per iteration.  The last
// CTA of each replica to finish a row kernel reduces that replica's partial
// sums in a fixed order (deterministic), decides its convergence on the
// device, and the last replica to decide sets the condition of the CUDA
// graph while-node that holds the loop, so a solve needs no host round trip.
//
// Precision forms: FP64 (the reference's arithmetic), and mixed: FP32
// storage, FFTs and Gamma0 until the update norm falls below max(tol, 2e-6)
// (phase 1), then FP64 iterations from that field to the requested tol
// (phase 2).  Norms and partial sums are FP64 in both.
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

#include <algorithm>
#include <mutex>
#include <vector>

#include "common.cuh"
#include "fft.cuh"
#include "tma.cuh"

namespace mgk {

const void* twiddles(int n, int prec);

constexpr int kAaMax = 8;  // deepest Anderson history
struct Ls2dAA;

struct Ls2dRep {
  int nx, ny, nyh, ld, tc;
  int row_items, col_items;
  long long N;
  // constitutive law: 0 linear (elasticity.py:12-18); 1 secant degradation
  // (law_a = d, law_b = k); 2 Rose (law_a = eta, law_b = floor fraction,
  // law_ps = 1 for plane stress); 3 Landau, law_ps = 1 for plane stress (lp: v1, v2, v3,
  // g1, g2, g3, g4, capping 0 none / 1 piecewise / 2 smooth, E_cap, tangent
  // ratio, smooth power)
  int law, law_ps;
  double law_a, law_b;
  double lp[11];
  FftLen fx64, fy64, fx32, fy32;
  double* mu;
  double* lam;
  double* eps;   // 3 planes
  double* ep;    // 3 planes
  double* epa;   // 2 planes or null
  float* mu32;   // mixed plans only
  float* lam32;
  float* eps32;
  float* ep32;
  void* spec;    // 3 planes of nx*ld complex (double2, or float2 in FP32 phases)
  // per call
  const double* init;
  double* out_eps;
  double* out_sig;
  double* out_e33;  // Landau plane stress: the out-of-plane strain per voxel (set_e33_out; may be null)
  double eb[4];
  double tol;
  int max_iter;
  int row_first, col_first;  // first work item of this replica in the call's maps
  // Anderson mixing of this call (null: none): state, the ring's dG slots
  // and its x (the mix is applied by the first row pass of each iterate and,
  // when the iteration cap ends the loop, by the output kernel)
  const Ls2dAA* aa;
  const double* aa_dG;
  double* aa_x;
};

struct Ls2dState {
  double mu0, lam0, Bc, inv2mu0;
  double ebar[3];
  double abar;
  double extra_d0, extra_n0;
  int iter;
  int phase_iter;
  int done;    // 0 active, 1 finished the current phase, 2 finished
  int status;
  double diff;
  double means[4];  // warm-start means (xx, xy, yx, yy)
  double out_eps_mean[4];
  double out_sig_mean[4];
};

struct Ls2dCtl {
  unsigned int n_active;  // replicas iterating at the start of the current body
  unsigned int decided;
  unsigned int still;
  unsigned int bodies;    // loop bodies run in the current phase (guard)
  int any;
  int error;              // a bounded wait gave up (MGK_TIMEOUT)
};

struct Ls2dAA {
  int k;          // valid difference columns, in slots 0 .. k-1
  int slot_next;  // ring slot of the next column
  int have_prev;  // a previous (f, g) pair exists
  int nmix;       // columns of the current mix (0: the plain step)
  unsigned int ctr;  // blocks of the update kernel done (self-resetting)
  int pad;
  double A[kAaMax][kAaMax];  // Gram matrix <dF_i, dF_j>
  double gamma[kAaMax];
};

// The Anderson mix x = g - dG gamma of voxel i's three strain planes (g in
// e), written to the plan's strain planes and the ring's x.
__device__ __forceinline__ void aa_mix_voxel(const Ls2dRep& R, long long i, int nmix, const double* gam, double* e) {
  const long long N = R.N, n3 = 3 * N;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    double sm = 0.0;
#pragma unroll
    for (int j = 0; j < kAaMax; ++j)
      if (j < nmix) sm += gam[j] * R.aa_dG[(size_t)j * n3 + c * N + i];
    e[c] -= sm;
    R.eps[c * N + i] = e[c];
    R.aa_x[c * N + i] = e[c];
  }
}

__device__ __forceinline__ int aa_load(const Ls2dRep& R, double* gam) {
  const int nmix = R.aa->nmix;
#pragma unroll
  for (int j = 0; j < kAaMax; ++j) gam[j] = j < nmix ? R.aa->gamma[j] : 0.0;
  return nmix;
}

constexpr double kMixedPhase1Tol = 2e-6;
constexpr int kMixedPhase1Cap = 64;

// --------------------------------------------------------------- helpers ---

// eps~^ = -Gamma0(n) : tau^ for symmetric tau (2D), n a unit vector.
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

template <typename TS> struct Fields;
template <> struct Fields<double> {
  static __device__ __forceinline__ const double* mu(const Ls2dRep& R) { return R.mu; }
  static __device__ __forceinline__ const double* lam(const Ls2dRep& R) { return R.lam; }
  static __device__ __forceinline__ double* eps(const Ls2dRep& R) { return R.eps; }
  static __device__ __forceinline__ const double* ep(const Ls2dRep& R) { return R.ep; }
  static __device__ __forceinline__ const FftLen& fx(const Ls2dRep& R) { return R.fx64; }
  static __device__ __forceinline__ const FftLen& fy(const Ls2dRep& R) { return R.fy64; }
};
template <> struct Fields<float> {
  static __device__ __forceinline__ const float* mu(const Ls2dRep& R) { return R.mu32; }
  static __device__ __forceinline__ const float* lam(const Ls2dRep& R) { return R.lam32; }
  static __device__ __forceinline__ float* eps(const Ls2dRep& R) { return R.eps32; }
  static __device__ __forceinline__ const float* ep(const Ls2dRep& R) { return R.ep32; }
  static __device__ __forceinline__ const FftLen& fx(const Ls2dRep& R) { return R.fx32; }
  static __device__ __forceinline__ const FftLen& fy(const Ls2dRep& R) { return R.fy32; }
};

// -------------------------------------------------------------- kernels ---

// Secant shear modulus mu (1 - d (1 - exp(-k eps_eq))) (elasticity.py:189-214)
// at the von Mises equivalent strain of the elastic strain (dxx, dyy, sym
// dxy): sqrt(2/3 eps':eps') with the plane-strain eps'_33 = -(dxx + dyy)/3
// (elasticity.py:112-150; the two shear entries sum to 2 dxy).
__device__ __forceinline__ double secant_mu(double m, double dxx, double dyy, double dxy, double d, double k) {
  const double tr3 = (dxx + dyy) / 3.0;
  const double a = dxx - tr3, b = dyy - tr3, c = -(dxx + dyy) / 3.0, sh = 2.0 * dxy;
  const double eq = sqrt((2.0 / 3.0) * (a * a + b * b + c * c + 0.5 * sh * sh));
  return m * (1.0 - d * (1.0 - exp(-k * eq)));
}

// Rose secant model (elasticity.py:868-944) at the elastic strain (dxx, dyy,
// dxy = its [0,1] entry): G = max(mu exp(-eta eq), floor mu), bulk modulus
// K = lam + 2 mu / 3 kept, lam_eff = K - 2 G / 3; plane stress solves
// eps_zz by the reference's five fixed-point steps.  Returns the trace
// (eps_zz included) and sets G and lam_eff.
__device__ __forceinline__ double rose_moduli(double l, double m, double dxx, double dyy, double dxy, double eta,
                                              double floor_f, int pstress, double& G, double& lam_eff) {
  const double K = l + (2.0 / 3.0) * m;
  double ezz = 0.0;
  auto eq_of = [&](double zz) {
    const double tr3 = (dxx + dyy + zz) / 3.0;
    const double a = dxx - tr3, b = dyy - tr3, c = zz - tr3;
    return sqrt((2.0 / 3.0) * (a * a + b * b + c * c + 2.0 * dxy * dxy));
  };
  auto g_of = [&](double eq) { return fmax(m * exp(-eta * eq), floor_f * m); };
  if (pstress) {
    ezz = -l / (l + 2.0 * m) * (dxx + dyy);
    for (int it = 0; it < 5; ++it) {
      const double g = g_of(eq_of(ezz));
      ezz = -((3.0 * K - 2.0 * g) / (3.0 * K + 4.0 * g)) * (dxx + dyy);
    }
  }
  G = g_of(eq_of(ezz));
  lam_eff = K - (2.0 / 3.0) * G;
  return dxx + dyy + ezz;
}

// Landau small-strain stress, plane strain (elasticity.py:487-639 with
// e33 = 0), parameters lp as in Ls2dRep; a12, a21 the two shear entries of
// the elastic strain.  With capping on, every voxel's strain goes through the
// capped form f (a - m) + m, as in the reference.
// Capped components, invariants and coefficients of the Landau law at the
// block-diagonal strain (in-plane a, out-of-plane e33)
// (elasticity.py:527-569).
struct LandauScal {
  double c11, c22, c12, c21, c33, w, I1, I2, cI, ce, ce2;
};

__device__ __forceinline__ LandauScal landau_scal(double mu, double lam, double a11, double a22, double a12,
                                                  double a21, double e33, const double* __restrict__ lp) {
  const double v1 = lp[0], v2 = lp[1], v3 = lp[2], g1 = lp[3], g2 = lp[4], g3 = lp[5], g4 = lp[6];
  const int cap = (int)lp[7];
  LandauScal s;
  s.c11 = a11; s.c22 = a22; s.c12 = a12; s.c21 = a21; s.c33 = e33; s.w = 0.0;
  if (cap) {
    const double m3 = (a11 + a22 + e33) / 3.0;
    const double d11 = a11 - m3, d22 = a22 - m3, d33 = e33 - m3;
    const double Ecap = lp[8];
    const double Eeq = sqrt(fmax(0.0, (2.0 / 3.0) * (d11 * d11 + d22 * d22 + d33 * d33 + 2.0 * a12 * a21)));
    double f = 1.0;
    if (cap == 2) {
      const double pw = lp[10];
      if (Eeq > 1e-12) f = (Ecap / Eeq) * pow(tanh(fmin(100.0, pow(Eeq / Ecap, pw))), 1.0 / pw);
      const double t = tanh(fmin(100.0, pow(Eeq / Ecap, pw)));
      s.w = t * t;
    } else if (Eeq > Ecap) {
      f = Ecap / Eeq;
      s.w = 1.0;
    }
    s.c11 = f * d11 + m3;
    s.c22 = f * d22 + m3;
    s.c12 = f * a12;
    s.c21 = f * a21;
    s.c33 = f * d33 + m3;
  }
  const double c11 = s.c11, c22 = s.c22, c33 = s.c33;
  const double I1 = c11 + c22 + c33;
  const double cross = s.c12 * s.c21;
  const double tr2 = c11 * c11 + c22 * c22 + 2.0 * cross;
  const double I2 = tr2 + c33 * c33;
  const double t_ip = c11 + c22;
  const double I3 = t_ip * (tr2 - (c11 * c22 - cross)) + c33 * c33 * c33;
  s.I1 = I1;
  s.I2 = I2;
  s.cI = lam * I1 + 0.5 * v1 * (I1 * I1) + v2 * I2 + (1.0 / 6.0) * g1 * (I1 * I1 * I1) + g2 * I1 * I2 +
         (4.0 / 3.0) * g3 * I3;
  s.ce = 2.0 * (mu + v2 * I1 + 0.5 * g2 * (I1 * I1) + g4 * I2);
  s.ce2 = 4.0 * (v3 + g3 * I1);
  return s;
}

// The Landau small-strain stress of a 2D voxel (elasticity.py:487-639).
// Plane strain: e33 = 0.  Plane stress (ps): e33 from the reference's Newton
// steps on sigma33 = 0 (:571-616) from the linear guess
// -lam/(lam + 2 mu) tr a, here until the voxel's step is below 1e-14 (at
// most 64 steps); the stress is evaluated at the stepped e33.  The
// reference runs the steps of all voxels together until every step is below
// 1e-9, evaluates each voxel before its last step and warm-starts the next
// call from the stepped field, so across its solver's iterations e33
// converges to the root of sigma33 = 0, which the kernel solves for at
// every evaluation.  With capping the step's derivative leaves out the
// capping factor's dependence on e33 and the steps converge linearly, so a
// single cold solve stopped at 1e-9 would leave ~1e-10 in e33.  e33_out
// (may be null) receives e33.
__device__ __forceinline__ void landau_sigma(double mu, double lam, double a11, double a22, double a12, double a21,
                                             const double* __restrict__ lp, int ps, double& s11, double& s22,
                                             double& s12, double& s21, double* e33_out = nullptr) {
  double e33 = 0.0;
  if (ps) {
    const double v1 = lp[0], v2 = lp[1], g1 = lp[3], g2 = lp[4], g3 = lp[5], g4 = lp[6];
    const double Gt = lp[9] * mu;
    e33 = -lam / (lam + 2.0 * mu) * (a11 + a22);
#pragma unroll 1
    for (int it = 0; it < 64; ++it) {
      const LandauScal t = landau_scal(mu, lam, a11, a22, a12, a21, e33, lp);
      const double c33 = t.c33, I1 = t.I1, I2 = t.I2;
      double s33 = t.cI + t.ce * c33 + t.ce2 * (c33 * c33);
      const double dcI = lam + v1 * I1 + 0.5 * g1 * (I1 * I1) + g2 * I2 + 2.0 * (v2 + g2 * I1) * c33 +
                         4.0 * g3 * (c33 * c33);
      const double dce = 2.0 * (v2 + g2 * I1) + 4.0 * g4 * c33;
      double ds33 = dcI + dce * c33 + t.ce + 4.0 * g3 * (c33 * c33) + 2.0 * t.ce2 * c33;
      if ((int)lp[7]) {
        s33 = s33 + 2.0 * Gt * (e33 - c33) * t.w;
        ds33 = ds33 + 2.0 * Gt * t.w;
      }
      const double delta = -s33 / (ds33 + 1e-12);
      e33 = e33 + delta;
      if (!(fabs(delta) >= 1e-14)) break;  // also leaves on NaN, which the stress then carries
    }
    if (e33_out) *e33_out = e33;
  }
  const LandauScal t = landau_scal(mu, lam, a11, a22, a12, a21, e33, lp);
  const double cross = t.c12 * t.c21;
  const double t_ip = t.c11 + t.c22;
  s11 = t.cI + t.ce * t.c11 + t.ce2 * (t.c11 * t.c11 + cross);
  s22 = t.cI + t.ce * t.c22 + t.ce2 * (t.c22 * t.c22 + cross);
  s12 = t.ce * t.c12 + t.ce2 * (t.c12 * t_ip);
  s21 = t.ce * t.c21 + t.ce2 * (t.c21 * t_ip);
  if ((int)lp[7]) {
    const double r = 2.0 * (lp[9] * mu) * t.w;
    s11 += r * (a11 - t.c11);
    s22 += r * (a22 - t.c22);
    s12 += r * (a12 - t.c12);
    s21 += r * (a21 - t.c21);
  }
}

// stress of the elastic strain (dxx, dyy, dxy) under law LAW; m, l the voxel's
// mu, lambda; LAW 0 is Hooke's law with the reference's operation order
template <int LAW>
__device__ __forceinline__ void law_sigma(double m, double l, double dxx, double dyy, double dxy, double a, double b,
                                          int ps, double& sxx, double& syy, double& sxy,
                                          const double* __restrict__ lp = nullptr) {
  if constexpr (LAW == 3) {
    double syx;
    landau_sigma(m, l, dxx, dyy, dxy, dxy, lp, ps, sxx, syy, sxy, syx);
  } else if constexpr (LAW == 2) {
    double G, le;
    const double tr = rose_moduli(l, m, dxx, dyy, dxy, a, b, ps, G, le);
    sxx = le * tr + 2.0 * G * dxx;
    syy = le * tr + 2.0 * G * dyy;
    sxy = 2.0 * G * dxy;
  } else {
    const double ms = LAW == 1 ? secant_mu(m, dxx, dyy, dxy, a, b) : m;
    const double trd = dxx + dyy;
    sxx = 2 * ms * dxx + l * trd;
    syy = 2 * ms * dyy + l * trd;
    sxy = 2 * ms * dxy;
  }
}

// Per-voxel material prep for one replica: mu, lambda from (E, nu) as in
// elasticity.py:3-10 (set_moduli 1), or given directly (set_moduli 2: E holds
// lambda, nu holds mu, as the secant solver takes them), eigenstrain planes
// (and FP32 copies for mixed plans), per-CTA partial sums of the two inputs
// for the reference medium.
__global__ void ls2d_material_kernel(const Ls2dRep* reps, int rep, const double* __restrict__ E,
                                     const double* __restrict__ nu, const double* __restrict__ epsp,
                                     int plane_mode, int set_moduli, double* partials) {
  __shared__ double red[32];
  const Ls2dRep& R = reps[rep];
  const long long N = R.N;
  double sE = 0, sn = 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N;
       i += (long long)gridDim.x * blockDim.x) {
    if (set_moduli) {
      const double e = E[i], v = nu[i];
      const double mu = set_moduli == 2 ? v : e / (2 * (1 + v));
      const double lam = set_moduli == 2 ? e
                         : plane_mode == MGK_PLANE_STRESS ? e * v / (1 - v * v)
                                                          : e * v / ((1 + v) * (1 - 2 * v));
      R.mu[i] = mu;
      R.lam[i] = lam;
      if (R.mu32) { R.mu32[i] = (float)mu; R.lam32[i] = (float)lam; }
      sE += e;
      sn += v;
    }
    double pxx = 0, pxy = 0, pyx = 0, pyy = 0;
    if (epsp) {
      const double4 p = reinterpret_cast<const double4*>(epsp)[i];
      pxx = p.x; pxy = p.y; pyx = p.z; pyy = p.w;
    }
    const double psym = (pxy == pyx) ? pxy : 0.5 * (pxy + pyx);
    R.ep[i] = pxx;
    R.ep[N + i] = pyy;
    R.ep[2 * N + i] = psym;
    if (R.ep32) { R.ep32[i] = (float)pxx; R.ep32[N + i] = (float)pyy; R.ep32[2 * N + i] = (float)psym; }
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

// Reference medium from the means: of E and nu (linear_elastic_simulator.py:
// 22-26), or of lambda and mu (lame_in 1: the secant solver, :679-681;
// lame_in 2: the Rose solver's (mean lambda, (mean mu + floor mean mu) / 2),
// :866-869).
__global__ void ls2d_medium_kernel(const Ls2dRep* reps, Ls2dState* st, int rep, const double* partials,
                                   int nblocks, int plane_mode, int lame_in, double floor_f) {
  __shared__ double red[32];
  double a = 0, b = 0;
  for (int i = threadIdx.x; i < nblocks; i += blockDim.x) { a += partials[2 * i]; b += partials[2 * i + 1]; }
  a = block_sum(a, red);
  b = block_sum(b, red);
  if (threadIdx.x == 0) {
    const double N = (double)reps[rep].N;
    const double E = a / N, v = b / N;
    const double mu0 = lame_in == 2 ? 0.5 * (v + floor_f * v) : lame_in ? v : E / (2 * (1 + v));
    const double lam0 = lame_in ? E
                        : plane_mode == MGK_PLANE_STRESS ? E * v / (1 - v * v) : E * v / ((1 + v) * (1 - 2 * v));
    Ls2dState& S = st[rep];
    S.mu0 = mu0;
    S.lam0 = lam0;
    S.Bc = (lam0 + mu0) / (mu0 * (lam0 + 2 * mu0));
    S.inv2mu0 = 1.0 / (2 * mu0);
  }
}

// Warm-start means: per-CTA partials of the 4 components of each selected
// replica's init field.  grid = (G, nsel).
__global__ void ls2d_means_kernel(const Ls2dRep* reps, const int* sel, double* partials) {
  __shared__ double red[32];
  const int r = sel[blockIdx.y];
  const Ls2dRep& R = reps[r];
  if (!R.init) return;
  const long long N = R.N;
  double s[4] = {0, 0, 0, 0};
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N;
       i += (long long)gridDim.x * blockDim.x) {
    const double4 v = reinterpret_cast<const double4*>(R.init)[i];
    s[0] += v.x; s[1] += v.y; s[2] += v.z; s[3] += v.w;
  }
  for (int q = 0; q < 4; ++q) {
    double t = block_sum(s[q], red);
    if (threadIdx.x == 0) partials[((size_t)blockIdx.y * gridDim.x + blockIdx.x) * 8 + q] = t;
  }
}

// Fixed-order sums of the per-CTA partials of replica sel[blockIdx.x]: K
// values at byte offset `off` of its state.  need_init: 0 -> means (scaled
// by 1/N) for every replica, 1 -> means only for replicas with a warm start,
// 2 -> plain sums only for replicas with a warm start.
__global__ void ls2d_finalize_kernel(const Ls2dRep* reps, Ls2dState* st, const int* sel, const double* partials,
                                     int G, int K, int off, int need_init) {
  __shared__ double red[32];
  const int r = sel[blockIdx.x];
  if (need_init && !reps[r].init) return;
  const double scale = need_init == 2 ? 1.0 : 1.0 / (double)reps[r].N;
  double* out = reinterpret_cast<double*>(reinterpret_cast<char*>(&st[r]) + off);
  for (int q = 0; q < K; ++q) {
    double a = 0;
    for (int i = threadIdx.x; i < G; i += blockDim.x) a += partials[((size_t)blockIdx.x * G + i) * 8 + q];
    a = block_sum(a, red);
    if (threadIdx.x == 0) out[q] = a * scale;
  }
}

// Solve start for each selected replica: eps_bar, caps and the initial field
// (linear_elastic_simulator.py:32-41), and partial sums of the antisymmetric
// part's contribution to the first diff and norm.  grid = (G, nsel).
__global__ void ls2d_begin_kernel(const Ls2dRep* reps, Ls2dState* st, const int* sel, double* partials) {
  __shared__ double red[32];
  const int r = sel[blockIdx.y];
  const Ls2dRep& R = reps[r];
  Ls2dState& S = st[r];
  const long long N = R.N;
  const double e00 = R.eb[0], e01 = R.eb[1], e10 = R.eb[2], e11 = R.eb[3];
  const double abar = 0.5 * (e01 - e10);
  const double sbar = (e01 == e10) ? e01 : 0.5 * (e01 + e10);
  const double* init = R.init;
  double d2 = 0, n2 = 0;
  double m00 = 0, m01 = 0, m10 = 0, m11 = 0;
  if (init) { m00 = S.means[0]; m01 = S.means[1]; m10 = S.means[2]; m11 = S.means[3]; }
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N;
       i += (long long)gridDim.x * blockDim.x) {
    double xx, yy, sy;
    if (init) {
      const double4 v = reinterpret_cast<const double4*>(init)[i];
      xx = v.x + (e00 - m00);
      const double xy = v.y + (e01 - m01), yx = v.z + (e10 - m10);
      yy = v.w + (e11 - m11);
      sy = (xy == yx) ? xy : 0.5 * (xy + yx);
      const double a0 = 0.5 * (xy - yx);
      d2 += 2 * (abar - a0) * (abar - a0);
      n2 += 2 * a0 * a0;
    } else {
      xx = e00; yy = e11; sy = sbar;
    }
    R.eps[i] = xx;
    R.eps[N + i] = yy;
    R.eps[2 * N + i] = sy;
    if (R.eps32) { R.eps32[i] = (float)xx; R.eps32[N + i] = (float)yy; R.eps32[2 * N + i] = (float)sy; }
  }
  if (init) {
    d2 = block_sum(d2, red);
    n2 = block_sum(n2, red);
    if (threadIdx.x == 0) {
      partials[((size_t)blockIdx.y * gridDim.x + blockIdx.x) * 8 + 0] = d2;
      partials[((size_t)blockIdx.y * gridDim.x + blockIdx.x) * 8 + 1] = n2;
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    S.ebar[0] = e00;
    S.ebar[1] = e11;
    S.ebar[2] = sbar;
    S.abar = abar;
    S.iter = 0;
    S.phase_iter = 0;
    S.done = R.max_iter <= 0 ? 2 : 0;
    S.status = MGK_OK;
    S.diff = 0;
    if (!init) { S.extra_d0 = 0; S.extra_n0 = 2.0 * (double)N * abar * abar; }
  }
}

// Convergence decision of replica r once the last of its row items has
// written its partial sums (all threads of the CTA call; thread 0 decides).
// The last replica to decide sets the graph while-node's condition.
template <bool FINAL>
__device__ void ls2d_decide(const Ls2dRep& R, Ls2dState& S, const double* partials, Ls2dCtl* ctl,
                            cudaGraphConditionalHandle cond, int use_cond, int guard_cap, double* red) {
  double a = 0, b = 0;
  for (int i = threadIdx.x; i < R.row_items; i += blockDim.x) {
    a += __ldcg(&partials[2 * (R.row_first + i)]);
    b += __ldcg(&partials[2 * (R.row_first + i) + 1]);
  }
  a = block_sum(a, red);
  b = block_sum(b, red);
  if (threadIdx.x != 0) return;
  if (S.iter == 0) { a += S.extra_d0; b += S.extra_n0; }
  else { b += 2.0 * (double)R.N * S.abar * S.abar; }
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
    const double tol1 = R.tol > kMixedPhase1Tol ? R.tol : kMixedPhase1Tol;
    if (S.iter >= R.max_iter) { S.done = 2; S.status = diff < R.tol ? MGK_OK : MGK_NOT_CONVERGED; }
    else if (diff < tol1 || S.phase_iter >= kMixedPhase1Cap) S.done = 1;
    else keep = 1;
  }
  const unsigned int n_act = ctl->n_active;  // stable until every active replica has decided
  if (keep) atomicAdd(&ctl->still, 1u);
  __threadfence();
  const unsigned int d = atomicAdd(&ctl->decided, 1u);
  if (d == n_act - 1) {
    __threadfence();
    const unsigned int still = atomicExch(&ctl->still, 0u);
    ctl->decided = 0;
    ctl->n_active = still;
    const bool go = still > 0 && atomicAdd(&ctl->bodies, 0u) <= (unsigned int)guard_cap && *(volatile int*)&ctl->error == 0;
    ctl->any = go ? 1 : 0;
    if (use_cond) cudaGraphSetConditional(cond, go ? 1u : 0u);
  }
}

// Row kernel.  IN_SPEC: the previous iteration's spectrum is inverted and the
// field updated (with diff/norm and the convergence decision); otherwise the
// field is read as is (first tau of a phase).  FINAL: this phase's decision
// is the last one (FP64 plans, or phase 2 of mixed plans).
template <typename TS, typename TC, bool IN_SPEC, bool FINAL>
__global__ void __launch_bounds__(256) ls2d_row_kernel(const Ls2dRep* __restrict__ reps, Ls2dState* st,
                                                      const int* __restrict__ row_map,
                                                      const int* __restrict__ row_local, double* partials,
                                                      unsigned int* rep_counter, Ls2dCtl* ctl,
                                                      cudaGraphConditionalHandle cond, int use_cond,
                                                      int guard_cap) {
  using C = C_t<TC>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ double red[32];
  __shared__ int s_last;
  const int item = blockIdx.x;
  const int r = row_map[item];
  const Ls2dRep& R = reps[r];
  Ls2dState& S = st[r];
  if (IN_SPEC && use_cond && item == 0 && threadIdx.x == 0) {
    // a body with no active replica has no decider: stop here; the body
    // count bounds the loop whatever happens to the deciders
    const unsigned int b = atomicAdd(&ctl->bodies, 1u) + 1u;
    if (ctl->n_active == 0 || b > (unsigned int)guard_cap || *(volatile int*)&ctl->error != 0) {
      ctl->any = 0;
      cudaGraphSetConditional(cond, 0u);
    }
  }
  if (S.done != 0) return;
  const int ny = R.ny, nyh = R.nyh, ld = R.ld, nx = R.nx;
  const long long N = R.N;
  const int x0 = 2 * row_local[item];
  C* bufA = reinterpret_cast<C*>(smem_raw);
  C* bufB = bufA + 3 * ny;
  C* spec = reinterpret_cast<C*>(R.spec);
  const double mu0 = S.mu0, lam0 = S.lam0;
  const int law = R.law, law_ps = R.law_ps;
  const double law_a = R.law_a, law_b = R.law_b;
  const double eb0 = S.ebar[0], eb1 = S.ebar[1], eb2 = S.ebar[2];
  TS* eps = Fields<TS>::eps(R);
  const TS* mu = Fields<TS>::mu(R);
  const TS* lam = Fields<TS>::lam(R);
  const TS* ep = Fields<TS>::ep(R);
  const FftLen& fy = Fields<TS>::fy(R);
  double d2 = 0, n2 = 0;
  C* cur = bufA;
  if (IN_SPEC) {
    const int tot = 3 * ny;
    for (int e0 = threadIdx.x; e0 < tot; e0 += 4 * blockDim.x) {
      C av[4], bv[4];
      int kk[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int e = e0 + u * blockDim.x;
        kk[u] = -1;
        if (e < tot) {
          const int c = e / ny, k = e - c * ny;
          const int ks = (2 * k <= ny) ? k : ny - k;
          const C* ra = spec + ((size_t)c * nx + x0) * ld;
          av[u] = ra[ks];
          bv[u] = ra[ld + ks];
          kk[u] = k;
        }
      }
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        if (kk[u] < 0) continue;
        const int e = e0 + u * blockDim.x, k = kk[u];
        C a = av[u], b = bv[u];
        C z;
        if (2 * k <= ny) {
          if (k == 0 || 2 * k == ny) { a.y = 0; b.y = 0; }
          z = mk<C>(a.x - b.y, a.y + b.x);
        } else {
          z = mk<C>(a.x + b.y, b.x - a.y);
        }
        bufA[e] = z;  // e = c * ny + k
      }
    }
    __syncthreads();
    cur = fft_any<+1>(bufA, bufB, 3, ny, fy);
  }
  C* out = (IN_SPEC && cur == bufA) ? bufB : bufA;
  double gam[kAaMax];
  const int nmix = (!IN_SPEC && sizeof(TS) == 8 && R.aa) ? aa_load(R, gam) : 0;
  // with Anderson mixing the image's tau is never used (see row_fast_body)
  const bool img_only = IN_SPEC && sizeof(TS) == 8 && law != 0 && R.aa != nullptr;
  for (int y = threadIdx.x; y < ny; y += blockDim.x) {
    TC tr[2][3];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const long long i = (long long)(x0 + h) * ny + y;
      double e[3];
      const double o0 = (double)eps[i], o1 = (double)eps[N + i], o2 = (double)eps[2 * N + i];
      const double m = (double)mu[i], l = (double)lam[i];
      const double p0 = (double)ep[i], p1 = (double)ep[N + i], p2 = (double)ep[2 * N + i];
      if (IN_SPEC) {
        const C z0 = cur[y], z1 = cur[ny + y], z2 = cur[2 * ny + y];
        e[0] = eb0 + (double)(h == 0 ? z0.x : z0.y);
        e[1] = eb1 + (double)(h == 0 ? z1.x : z1.y);
        e[2] = eb2 + (double)(h == 0 ? z2.x : z2.y);
        const double q0 = e[0] - o0, q1 = e[1] - o1, q2 = e[2] - o2;
        d2 += q0 * q0 + q1 * q1 + 2.0 * q2 * q2;
        n2 += o0 * o0 + o1 * o1 + 2.0 * o2 * o2;
        eps[i] = (TS)e[0];
        eps[N + i] = (TS)e[1];
        eps[2 * N + i] = (TS)e[2];
      } else {
        e[0] = o0; e[1] = o1; e[2] = o2;
        if (!IN_SPEC && sizeof(TS) == 8 && R.aa) aa_mix_voxel(R, i, nmix, gam, e);  // the mixed iterate
      }
      if (img_only) continue;
      const double dxx = e[0] - p0, dyy = e[1] - p1, dxy = e[2] - p2;
      const double tre = e[0] + e[1];
      double s0, s1, s2;  // nonlinear laws only in FP64 kernels (their plans are FP64)
      if (sizeof(TS) == 8 && law == 1) law_sigma<1>(m, l, dxx, dyy, dxy, law_a, law_b, law_ps, s0, s1, s2);
      else if (sizeof(TS) == 8 && law == 2) law_sigma<2>(m, l, dxx, dyy, dxy, law_a, law_b, law_ps, s0, s1, s2);
      else if (sizeof(TS) == 8 && law == 3) law_sigma<3>(m, l, dxx, dyy, dxy, 0.0, 0.0, law_ps, s0, s1, s2, R.lp);
      else law_sigma<0>(m, l, dxx, dyy, dxy, 0.0, 0.0, 0, s0, s1, s2);
      tr[h][0] = (TC)(s0 - (2 * mu0 * e[0] + lam0 * tre));
      tr[h][1] = (TC)(s1 - (2 * mu0 * e[1] + lam0 * tre));
      tr[h][2] = (TC)(s2 - 2 * mu0 * e[2]);
    }
    if (img_only) continue;
#pragma unroll
    for (int c = 0; c < 3; ++c) out[c * ny + y] = mk<C>(tr[0][c], tr[1][c]);
  }
  if (!img_only) {
    __syncthreads();
    C* scratch = (out == bufA) ? bufB : bufA;
    C* Z = fft_any<-1>(out, scratch, 3, ny, fy);
    for (int e = threadIdx.x; e < 3 * nyh; e += blockDim.x) {
      const int c = e / nyh, k = e - c * nyh;
      const C z = Z[c * ny + k];
      const C w = Z[c * ny + (k == 0 ? 0 : ny - k)];
      C* ra = spec + ((size_t)c * nx + x0) * ld;
      ra[k] = mk<C>(TC(0.5) * (z.x + w.x), TC(0.5) * (z.y - w.y));
      ra[ld + k] = mk<C>(TC(0.5) * (z.y + w.y), TC(-0.5) * (z.x - w.x));
    }
  }
  if (!IN_SPEC) return;
  // partial sums -> fixed slot; the replica's last CTA reduces and decides
  d2 = block_sum(d2, red);
  n2 = block_sum(n2, red);
  if (threadIdx.x == 0) {
    partials[2 * item] = d2;
    partials[2 * item + 1] = n2;
    __threadfence();
    const unsigned int t = atomicInc(&rep_counter[r], (unsigned int)R.row_items - 1);  // self-resetting
    s_last = (t == (unsigned int)R.row_items - 1);
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  ls2d_decide<FINAL>(R, S, partials, ctl, cond, use_cond, guard_cap, red);
}

// Persistent row kernel (IN_SPEC iterations) with double-buffered bulk
// prefetch: each CTA walks the items blockIdx.x, +gridDim.x, ...; while it
// transforms one row pair, the inputs of its next row pair (two spectrum rows
// and two rows of eps, mu, lambda, eps_p, all contiguous) stream into the
// other shared-memory stage through cp.async.bulk.  Requires ny even (16-byte
// aligned rows).  Stage layout (bytes): spec [3][2][ld] C | eps [3][2][ny] |
// mu [2][ny] | lam [2][ny] | ep [3][2][ny] (TS).
template <typename TS, typename TC, bool FINAL>
__global__ void __launch_bounds__(256, 1) ls2d_row_tma_kernel(const Ls2dRep* __restrict__ reps, Ls2dState* st,
                                                             const int* __restrict__ row_map,
                                                             const int* __restrict__ row_local, double* partials,
                                                             unsigned int* rep_counter, Ls2dCtl* ctl,
                                                             cudaGraphConditionalHandle cond, int use_cond,
                                                             int guard_cap, int nitems, int stage_bytes) {
  using C = C_t<TC>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ double red[32];
  __shared__ int s_last;
  __shared__ __align__(8) uint64_t bars[2];
  C* bufA = reinterpret_cast<C*>(smem_raw + 2 * (size_t)stage_bytes);
  if (threadIdx.x == 0) {
    mbar_init(&bars[0], 1);
    mbar_init(&bars[1], 1);
    fence_mbar_init();
  }
  if (use_cond && blockIdx.x == 0 && threadIdx.x == 0) {
    const unsigned int b = atomicAdd(&ctl->bodies, 1u) + 1u;
    if (ctl->n_active == 0 || b > (unsigned int)guard_cap || *(volatile int*)&ctl->error != 0) {
      ctl->any = 0;
      cudaGraphSetConditional(cond, 0u);
    }
  }
  __syncthreads();
  uint32_t parity[2] = {0u, 0u};
  // issue the bulk loads of `item` into stage s; returns whether it is active
  auto issue = [&](int item, int s) -> bool {
    const int r = row_map[item];
    if (st[r].done != 0) return false;
    if (threadIdx.x == 0) {
      const Ls2dRep& R = reps[r];
      const int ny = R.ny, ld = R.ld;
      const long long N = R.N;
      const long long x0 = 2LL * row_local[item];
      unsigned char* sb = smem_raw + (size_t)s * stage_bytes;
      const uint32_t spec_b = 2u * ld * sizeof(C), row_b = 2u * ny * sizeof(TS);
      // the copy list in stage order; the barrier expects exactly its bytes
      const void* src[11];
      uint32_t len[11];
      int n = 0;
      const C* spec = reinterpret_cast<const C*>(R.spec);
      for (int c = 0; c < 3; ++c) { src[n] = spec + ((long long)c * R.nx + x0) * ld; len[n++] = spec_b; }
      const TS* eps = Fields<TS>::eps(R);
      const TS* ep = Fields<TS>::ep(R);
      for (int c = 0; c < 3; ++c) { src[n] = eps + c * N + x0 * ny; len[n++] = row_b; }
      src[n] = Fields<TS>::mu(R) + x0 * ny; len[n++] = row_b;
      src[n] = Fields<TS>::lam(R) + x0 * ny; len[n++] = row_b;
      for (int c = 0; c < 3; ++c) { src[n] = ep + c * N + x0 * ny; len[n++] = row_b; }
      uint32_t total = 0;
      for (int q = 0; q < n; ++q) total += len[q];
      fence_proxy_async_smem();
      mbar_arrive_expect_tx(&bars[s], total);
      unsigned char* dst = sb;
      for (int q = 0; q < n; ++q) { bulk_g2s(dst, src[q], len[q], &bars[s]); dst += len[q]; }
    }
    return true;
  };
  int item = blockIdx.x;
  bool act = item < nitems ? issue(item, 0) : false;
  for (int k = 0; item < nitems; item += gridDim.x, ++k) {
    const int s = k & 1;
    const int next = item + gridDim.x;
    const bool act_next = next < nitems ? issue(next, s ^ 1) : false;
    if (act) {
      const bool ok = __syncthreads_and(mbar_wait(&bars[s], parity[s]) ? 1 : 0);
      parity[s] ^= 1u;
      if (!ok) {
        // the copy never completed: record it, wait (bounded) for the other
        // stage's copy if one is in flight, and leave
        if (threadIdx.x == 0) { ctl->error = 1; ctl->any = 0; }
        if (act_next) mbar_wait(&bars[s ^ 1], parity[s ^ 1]);
        return;
      }
      const int r = row_map[item];
      const Ls2dRep& R = reps[r];
      Ls2dState& S = st[r];
      const int ny = R.ny, nyh = R.nyh, ld = R.ld, nx = R.nx;
      const long long N = R.N;
      const int x0 = 2 * row_local[item];
      unsigned char* sb = smem_raw + (size_t)s * stage_bytes;
      const uint32_t spec_b = 2u * ld * sizeof(C), row_b = 2u * ny * sizeof(TS);
      const C* sspec = reinterpret_cast<const C*>(sb);
      const TS* seps = reinterpret_cast<const TS*>(sb + 3 * spec_b);
      const TS* smu = reinterpret_cast<const TS*>(sb + 3 * spec_b + 3 * row_b);
      const TS* slam = smu + 2 * ny;
      const TS* sep = slam + 2 * ny;
      const FftLen& fy = Fields<TS>::fy(R);
      for (int e = threadIdx.x; e < 3 * ny; e += blockDim.x) {
        const int c = e / ny, k2 = e - c * ny;
        const int ks = (2 * k2 <= ny) ? k2 : ny - k2;
        C a = sspec[c * 2 * ld + ks], b = sspec[c * 2 * ld + ld + ks];
        C z;
        if (2 * k2 <= ny) {
          if (k2 == 0 || 2 * k2 == ny) { a.y = 0; b.y = 0; }
          z = mk<C>(a.x - b.y, a.y + b.x);
        } else {
          z = mk<C>(a.x + b.y, b.x - a.y);
        }
        bufA[e] = z;
      }
      __syncthreads();
      C* bufB = reinterpret_cast<C*>(sb);  // the spectrum rows are consumed
      C* cur = fft_any<+1>(bufA, bufB, 3, ny, fy);
      C* out = (cur == bufA) ? bufB : bufA;
      const double mu0 = S.mu0, lam0 = S.lam0;
      const int law = R.law, law_ps = R.law_ps;
  const double law_a = R.law_a, law_b = R.law_b;
      const double eb0 = S.ebar[0], eb1 = S.ebar[1], eb2 = S.ebar[2];
      TS* eps = Fields<TS>::eps(R);
      double d2 = 0, n2 = 0;
      for (int y = threadIdx.x; y < ny; y += blockDim.x) {
        TC tr[2][3];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int j = h * ny + y;
          const long long i = (long long)(x0 + h) * ny + y;
          const double o0 = (double)seps[j], o1 = (double)seps[2 * ny + j], o2 = (double)seps[4 * ny + j];
          const double m = (double)smu[j], l = (double)slam[j];
          const double p0 = (double)sep[j], p1 = (double)sep[2 * ny + j], p2 = (double)sep[4 * ny + j];
          const C z0 = cur[y], z1 = cur[ny + y], z2 = cur[2 * ny + y];
          const double e0 = eb0 + (double)(h == 0 ? z0.x : z0.y);
          const double e1 = eb1 + (double)(h == 0 ? z1.x : z1.y);
          const double e2 = eb2 + (double)(h == 0 ? z2.x : z2.y);
          const double q0 = e0 - o0, q1 = e1 - o1, q2 = e2 - o2;
          d2 += q0 * q0 + q1 * q1 + 2.0 * q2 * q2;
          n2 += o0 * o0 + o1 * o1 + 2.0 * o2 * o2;
          eps[i] = (TS)e0;
          eps[N + i] = (TS)e1;
          eps[2 * N + i] = (TS)e2;
          const double dxx = e0 - p0, dyy = e1 - p1, dxy = e2 - p2;
          const double tre = e0 + e1;
          double s0, s1, s2;  // nonlinear laws only in FP64 kernels (their plans are FP64)
          if (sizeof(TS) == 8 && law == 1) law_sigma<1>(m, l, dxx, dyy, dxy, law_a, law_b, law_ps, s0, s1, s2);
          else if (sizeof(TS) == 8 && law == 2) law_sigma<2>(m, l, dxx, dyy, dxy, law_a, law_b, law_ps, s0, s1, s2);
          else if (sizeof(TS) == 8 && law == 3) law_sigma<3>(m, l, dxx, dyy, dxy, 0.0, 0.0, law_ps, s0, s1, s2, R.lp);
          else law_sigma<0>(m, l, dxx, dyy, dxy, 0.0, 0.0, 0, s0, s1, s2);
          tr[h][0] = (TC)(s0 - (2 * mu0 * e0 + lam0 * tre));
          tr[h][1] = (TC)(s1 - (2 * mu0 * e1 + lam0 * tre));
          tr[h][2] = (TC)(s2 - 2 * mu0 * e2);
        }
#pragma unroll
        for (int c = 0; c < 3; ++c) out[c * ny + y] = mk<C>(tr[0][c], tr[1][c]);
      }
      __syncthreads();
      C* scratch = (out == bufA) ? bufB : bufA;
      C* Z = fft_any<-1>(out, scratch, 3, ny, fy);
      C* spec = reinterpret_cast<C*>(R.spec);
      for (int e = threadIdx.x; e < 3 * nyh; e += blockDim.x) {
        const int c = e / nyh, k2 = e - c * nyh;
        const C z = Z[c * ny + k2];
        const C w = Z[c * ny + (k2 == 0 ? 0 : ny - k2)];
        C* ra = spec + ((size_t)c * nx + x0) * ld;
        ra[k2] = mk<C>(TC(0.5) * (z.x + w.x), TC(0.5) * (z.y - w.y));
        ra[ld + k2] = mk<C>(TC(0.5) * (z.y + w.y), TC(-0.5) * (z.x - w.x));
      }
      d2 = block_sum(d2, red);
      n2 = block_sum(n2, red);
      if (threadIdx.x == 0) {
        partials[2 * item] = d2;
        partials[2 * item + 1] = n2;
        __threadfence();
        const unsigned int t = atomicInc(&rep_counter[r], (unsigned int)R.row_items - 1);
        s_last = (t == (unsigned int)R.row_items - 1);
      }
      __syncthreads();
      if (s_last) {
        __threadfence();
        ls2d_decide<FINAL>(R, S, partials, ctl, cond, use_cond, guard_cap, red);
      }
    }
    __syncthreads();  // this stage is free for the prefetch two items ahead
    act = act_next;
  }
}

// Column kernel: FFT along x, Gamma0_sym, inverse FFT along x, for a tile of
// tc consecutive ky columns and all three components.
template <typename TS, typename TC>
__global__ void __launch_bounds__(256) ls2d_col_kernel(const Ls2dRep* __restrict__ reps,
                                                      const Ls2dState* __restrict__ st,
                                                      const int* __restrict__ col_map,
                                                      const int* __restrict__ col_local) {
  using C = C_t<TC>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int item = blockIdx.x;
  const int r = col_map[item];
  const Ls2dRep& R = reps[r];
  const Ls2dState& S = st[r];
  if (S.done != 0) return;
  const int nx = R.nx, ny = R.ny, nyh = R.nyh, ld = R.ld, tc = R.tc;
  const int ky0 = col_local[item] * tc;
  const int tcw = min(tc, nyh - ky0);
  const FftLen& fx = Fields<TS>::fx(R);
  C* bufA = reinterpret_cast<C*>(smem_raw);
  C* bufB = bufA + 3 * tc * nx;
  C* spec = reinterpret_cast<C*>(R.spec);
  const int tot = 3 * tcw * nx;
  for (int e0 = threadIdx.x; e0 < tot; e0 += 4 * blockDim.x) {
    C v[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int e = e0 + u * blockDim.x;
      if (e < tot) {
        const int c = e / (tcw * nx);
        const int rem = e - c * tcw * nx;
        const int x = rem / tcw, t = rem - x * tcw;
        v[u] = spec[((size_t)c * nx + x) * ld + ky0 + t];
      }
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int e = e0 + u * blockDim.x;
      if (e < tot) {
        const int c = e / (tcw * nx);
        const int rem = e - c * tcw * nx;
        const int x = rem / tcw, t = rem - x * tcw;
        bufA[(c * tc + t) * nx + x] = v[u];
      }
    }
  }
  __syncthreads();
  // lines (c * tc + t); only t < tcw are meaningful, all 3*tc are transformed
  C* F = fft_any<-1>(bufA, bufB, 3 * tc, nx, fx);
  const TC inv2mu0 = (TC)S.inv2mu0, Bc = (TC)S.Bc;
  const TC sc = (TC)(1.0 / ((double)nx * (double)ny));
  for (int e = threadIdx.x; e < tcw * nx; e += blockDim.x) {
    const int t = e / nx, kx = e - t * nx;
    const int ky = ky0 + t;
    C* pxx = &F[(0 * tc + t) * nx + kx];
    C* pyy = &F[(1 * tc + t) * nx + kx];
    C* pxy = &F[(2 * tc + t) * nx + kx];
    if (kx == 0 && ky == 0) {
      *pxx = mk<C>(TC(0), TC(0)); *pyy = *pxx; *pxy = *pxx;
      continue;
    }
    // fftfreq signs matter where several axes sit on their Nyquist line
    const double ux = (double)fftfreq(kx, nx) / nx, uy = (double)fftfreq(ky, ny) / ny;
    const double inv = 1.0 / sqrt(ux * ux + uy * uy);
    const TC nxv = (TC)(ux * inv), nyv = (TC)(uy * inv);
    const C txx = *pxx, tyy = *pyy, txy = *pxy;
    C exx, eyy, exy;
    gamma2d_apply(txx, tyy, txy, nxv, nyv, inv2mu0, Bc, exx, eyy, exy);
    const bool nqx = (nx & 1) == 0 && 2 * kx == nx, nqy = (ny & 1) == 0 && 2 * ky == ny;
    if (nqx || nqy) {
      C fxx, fyy, fxy;
      gamma2d_apply(txx, tyy, txy, nqx ? -nxv : nxv, nqy ? -nyv : nyv, inv2mu0, Bc, fxx, fyy, fxy);
      exx = mk<C>(TC(0.5) * (exx.x + fxx.x), TC(0.5) * (exx.y + fxx.y));
      eyy = mk<C>(TC(0.5) * (eyy.x + fyy.x), TC(0.5) * (eyy.y + fyy.y));
      exy = mk<C>(TC(0.5) * (exy.x + fxy.x), TC(0.5) * (exy.y + fxy.y));
    }
    *pxx = mk<C>(exx.x * sc, exx.y * sc);
    *pyy = mk<C>(eyy.x * sc, eyy.y * sc);
    *pxy = mk<C>(exy.x * sc, exy.y * sc);
  }
  __syncthreads();
  C* G = (F == bufA) ? bufB : bufA;
  C* Rz = fft_any<+1>(F, G, 3 * tc, nx, fx);
  for (int e = threadIdx.x; e < tot; e += blockDim.x) {
    const int c = e / (tcw * nx);
    const int rem = e - c * tcw * nx;
    const int x = rem / tcw, t = rem - x * tcw;
    spec[((size_t)c * nx + x) * ld + ky0 + t] = Rz[(c * tc + t) * nx + x];
  }
}

// --------------------------------------------- warp-line iteration kernels ---
// The same two stages for replicas whose sides have a compiled warp-line FFT
// (64 .. 512).  Row kernel: one CTA of three warps per pair of x-rows; one
// elected thread stages the pair's eps, mu, lambda and eps_p rows in shared
// memory with bulk asynchronous copies at entry, while warp c inverts
// component c of the spectrum; after one CTA barrier every thread updates its
// voxels and builds tau, then warp c forward-transforms and stores component
// c.  Column kernel: one CTA of kColTiles warps per tile of kColTiles ky
// columns; the tile lands in shared memory through cp.async, then warp t runs
// FFT, Gamma0_sym and inverse FFT on column t alone.
// resident-CTA targets for the register allocator (FP32 kernels need fewer
// registers; more resident warps hide their latency)
#ifndef MGK_ROW_MINB32
#define MGK_ROW_MINB32 9
#endif
#ifndef MGK_COL_MINB32
#define MGK_COL_MINB32 4
#endif
constexpr int kColTiles = 4;  // ky columns per column-kernel CTA (one warp each)
// lanes per line and column tiles of a kernel variant (sides up to MAXN):
// lines longer than 512 points take two warps
__host__ __device__ constexpr int fast_group(int maxn) { return maxn > 512 ? 64 : 32; }
__host__ __device__ constexpr int fast_col_tiles(int maxn) { return maxn > 512 ? 2 : kColTiles; }
__host__ __device__ constexpr int row_threads(int maxn) { return 3 * fast_group(maxn); }
__host__ __device__ constexpr int col_threads(int maxn) { return fast_col_tiles(maxn) * fast_group(maxn); }

// Shared memory of the row kernel: 3 padded lines, then the row pair's eps
// (3), mu, lambda and eps_p (3) planes staged by bulk copies (reading eps
// from global memory instead serialises the loads behind the in-place stores).
__host__ __device__ constexpr int row_fast_smem(int ny, int csz, int tsz) {
  return ((3 * (csz == 16 ? ny + ny / 8 + 1 : ((ny + ny / 16 + 2) & ~1)) * csz + 127) / 128) * 128 + 16 * ny * tsz;
}
__host__ __device__ constexpr int col_fast_smem(int nx, int csz, int tc) {
  return 3 * tc * (csz == 16 ? nx + nx / 8 + 1 : ((nx + nx / 16 + 2) & ~1)) * csz;
}

template <typename T, int NY, int G, bool IN_SPEC, bool FINAL, int LAW>
__device__ __forceinline__ void row_fast_body(const Ls2dRep& R, Ls2dState& S, int item, int r, int x0,
                                              double* partials,
                                              unsigned int* rep_counter, Ls2dCtl* ctl,
                                              cudaGraphConditionalHandle cond, int use_cond, int guard_cap,
                                              unsigned char* smem, uint64_t* bar, double* red, int* s_last) {
  using C = C_t<T>;
  constexpr int PL = padded_len<C>(NY);
  constexpr int NYH = NY / 2 + 1;
  constexpr int NT = 3 * G;
  const int warp = threadIdx.x / G, lane = threadIdx.x % G;  // line (component) and lane in it
  const int bid = 1 + warp;
  const int nx = R.nx, ld = R.ld;
  const long long N = R.N;
  C* lines = reinterpret_cast<C*>(smem);
  T* stg = reinterpret_cast<T*>(smem + ((3 * PL * (int)sizeof(C) + 127) / 128) * 128);
  T* eps = Fields<T>::eps(R);
  const T* ep = Fields<T>::ep(R);
  constexpr uint32_t rb = 2u * NY * sizeof(T);
  if (threadIdx.x == 0) {
    const T* src[8] = {eps, eps + N, eps + 2 * N, Fields<T>::mu(R), Fields<T>::lam(R), ep, ep + N, ep + 2 * N};
    fence_proxy_async_smem();
    mbar_arrive_expect_tx(bar, 8u * rb);
#pragma unroll
    for (int q = 0; q < 8; ++q) bulk_g2s(stg + q * 2 * NY, src[q] + (long long)x0 * NY, rb, bar);
  }
  const C* tw = reinterpret_cast<const C*>(Fields<T>::fy(R).tw);
  C* spec = reinterpret_cast<C*>(R.spec);
  C* line = lines + warp * PL;
  C* ra = spec + ((size_t)warp * nx + x0) * ld;
  C* rbp = ra + ld;
  if (IN_SPEC) {
    constexpr int U = (NYH + G - 1) / G;
    C a[U], b[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int k = lane + G * u;
      if (k < NYH) { a[u] = ra[k]; b[u] = rbp[k]; }
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int k = lane + G * u;
      if (k < NYH) {
        C av = a[u], bv = b[u];
        if (k == 0 || 2 * k == NY) { av.y = 0; bv.y = 0; }
        line[pidx<C>(k)] = mk<C>(av.x - bv.y, av.y + bv.x);
        if (k > 0 && 2 * k < NY) line[pidx<C>(NY - k)] = mk<C>(av.x + bv.y, bv.x - av.y);
      }
    }
    grp_sync<G>(bid);
    warp_fft<NY, +1, 1, G>(line, PL, tw, lane, bid);
  }
  const bool ok = mbar_wait(bar, 0);
  if (!__syncthreads_and(ok ? 1 : 0)) {
    if (threadIdx.x == 0) { ctl->error = 1; ctl->any = 0; }
    return;
  }
  const double mu0 = S.mu0, lam0 = S.lam0;
  const int law = R.law, law_ps = R.law_ps;
  const double law_a = R.law_a, law_b = R.law_b;
  const double eb0 = S.ebar[0], eb1 = S.ebar[1], eb2 = S.ebar[2];
  double gam[kAaMax];
  const int nmix = (!IN_SPEC && sizeof(T) == 8 && R.aa) ? aa_load(R, gam) : 0;
  // with Anderson mixing the image's tau is never used (the next tau is the
  // mixed iterate's): the pass stops at the image and its update norm
  const bool img_only = IN_SPEC && LAW != 0 && sizeof(T) == 8 && R.aa != nullptr;
  double d2 = 0, n2 = 0;
  for (int y = threadIdx.x; y < NY; y += NT) {
    T tr[2][3];
    const int py = pidx<C>(y);
    C z[3];
    if (IN_SPEC) {
#pragma unroll
      for (int c = 0; c < 3; ++c) z[c] = lines[c * PL + py];
    }
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int j = h * NY + y;
      const long long i = (long long)(x0 + h) * NY + y;
      const double o0 = (double)stg[j], o1 = (double)stg[2 * NY + j], o2 = (double)stg[4 * NY + j];
      const double m = (double)stg[6 * NY + j], l = (double)stg[8 * NY + j];
      const double p0 = (double)stg[10 * NY + j], p1 = (double)stg[12 * NY + j], p2 = (double)stg[14 * NY + j];
      double e0, e1, e2;
      if (IN_SPEC) {
        e0 = eb0 + (double)(h == 0 ? z[0].x : z[0].y);
        e1 = eb1 + (double)(h == 0 ? z[1].x : z[1].y);
        e2 = eb2 + (double)(h == 0 ? z[2].x : z[2].y);
        const double q0 = e0 - o0, q1 = e1 - o1, q2 = e2 - o2;
        d2 += q0 * q0 + q1 * q1 + 2.0 * q2 * q2;
        n2 += o0 * o0 + o1 * o1 + 2.0 * o2 * o2;
        eps[i] = (T)e0;
        eps[N + i] = (T)e1;
        eps[2 * N + i] = (T)e2;
      } else {
        e0 = o0; e1 = o1; e2 = o2;
        if (!IN_SPEC && sizeof(T) == 8 && R.aa) {  // the mixed iterate
          double e[3] = {o0, o1, o2};
          aa_mix_voxel(R, i, nmix, gam, e);
          e0 = e[0]; e1 = e[1]; e2 = e[2];
        }
      }
      if (img_only) continue;
      const double dxx = e0 - p0, dyy = e1 - p1, dxy = e2 - p2;
      const double tre = e0 + e1;
      double s0, s1, s2;  // LAW 0 linear; 1 secant, 2 Rose, 3 Landau (FP64 plans)
      law_sigma<LAW>(m, l, dxx, dyy, dxy, law_a, law_b, law_ps, s0, s1, s2, R.lp);
      tr[h][0] = (T)(s0 - (2 * mu0 * e0 + lam0 * tre));
      tr[h][1] = (T)(s1 - (2 * mu0 * e1 + lam0 * tre));
      tr[h][2] = (T)(s2 - 2 * mu0 * e2);
    }
    if (img_only) continue;
#pragma unroll
    for (int c = 0; c < 3; ++c) lines[c * PL + py] = mk<C>(tr[0][c], tr[1][c]);
  }
  if (!img_only) {
    __syncthreads();
    warp_fft<NY, -1, 1, G>(line, PL, tw, lane, bid);
    for (int k = lane; k < NYH; k += G) {
      const C zz = line[pidx<C>(k)];
      const C w = line[pidx<C>(k == 0 ? 0 : NY - k)];
      ra[k] = mk<C>(T(0.5) * (zz.x + w.x), T(0.5) * (zz.y - w.y));
      rbp[k] = mk<C>(T(0.5) * (zz.y + w.y), T(-0.5) * (zz.x - w.x));
    }
  }
  if (!IN_SPEC) return;
  d2 = block_sum(d2, red);
  n2 = block_sum(n2, red);
  if (threadIdx.x == 0) {
    partials[2 * item] = d2;
    partials[2 * item + 1] = n2;
    __threadfence();
    const unsigned int t = atomicInc(&rep_counter[r], (unsigned int)R.row_items - 1);  // self-resetting
    *s_last = (t == (unsigned int)R.row_items - 1);
  }
  __syncthreads();
  if (!*s_last) return;
  __threadfence();
  ls2d_decide<FINAL>(R, S, partials, ctl, cond, use_cond, guard_cap, red);
}

template <typename T, int MAXN, bool IN_SPEC, bool FINAL, int LAW = 0>
__global__ void __launch_bounds__(row_threads(MAXN), sizeof(T) == 4 && MAXN <= 256 ? MGK_ROW_MINB32 : 1) ls2d_row_fast_kernel(
    const Ls2dRep* __restrict__ reps, Ls2dState* st, const int* __restrict__ row_map,
    const int* __restrict__ row_local, double* partials, unsigned int* rep_counter, Ls2dCtl* ctl,
    cudaGraphConditionalHandle cond, int use_cond, int guard_cap) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ double red[32];
  __shared__ int s_last;
  __shared__ __align__(8) uint64_t bar;
  const int item = blockIdx.x;
  const int r = row_map[item];
  const Ls2dRep& R = reps[r];
  Ls2dState& S = st[r];
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
  const int x0 = 2 * row_local[item];
#define MGK_ROW_CASE(n) \
  case n: if constexpr (n <= MAXN) row_fast_body<T, n, fast_group(MAXN), IN_SPEC, FINAL, LAW>(R, S, item, r, x0, partials, rep_counter, ctl, cond, use_cond, guard_cap, \
                                              smem_raw, &bar, red, &s_last); break;
  switch (R.ny) {
    MGK_ROW_CASE(64) MGK_ROW_CASE(96) MGK_ROW_CASE(128) MGK_ROW_CASE(192) MGK_ROW_CASE(256) MGK_ROW_CASE(384)
    MGK_ROW_CASE(512) MGK_ROW_CASE(768) MGK_ROW_CASE(1024)
    default: break;
  }
#undef MGK_ROW_CASE
}

template <typename T, int NX, int TC, int G>
__device__ __forceinline__ void col_fast_body(const Ls2dRep& R, const Ls2dState& S, int ky0,
                                              unsigned char* smem) {
  using C = C_t<T>;
  constexpr int kColTiles = TC;
  constexpr int PL = padded_len<C>(NX);
  const int warp = threadIdx.x / G, lane = threadIdx.x % G;  // column of the tile and lane in it
  const int bid = 1 + warp;
  const int ny = R.ny, nyh = R.nyh, ld = R.ld;
  const int tcw = min(kColTiles, nyh - ky0);
  C* lines = reinterpret_cast<C*>(smem);  // line (c * kColTiles + t)
  C* spec = reinterpret_cast<C*>(R.spec);
  constexpr int TOT = 3 * NX * kColTiles;
  for (int e = threadIdx.x; e < TOT; e += G * kColTiles) {
    const int c = e / (NX * kColTiles);
    const int rem = e - c * NX * kColTiles;
    const int x = rem / kColTiles, t = rem - x * kColTiles;
    if (t < tcw) cp_async_elem(&lines[(c * kColTiles + t) * PL + pidx<C>(x)], &spec[((size_t)c * NX + x) * ld + ky0 + t]);
  }
  cp_async_wait_all();
  __syncthreads();
  const int t = warp;
  if (t < tcw) {
    const C* tw = reinterpret_cast<const C*>(Fields<T>::fx(R).tw);
    C* l0 = lines + t * PL;
    constexpr int LS = kColTiles * PL;  // stride between the components of a column
    warp_fft<NX, -1, 1, G>(l0, LS, tw, lane, bid);
    warp_fft<NX, -1, 1, G>(l0 + LS, LS, tw, lane, bid);
    warp_fft<NX, -1, 1, G>(l0 + 2 * LS, LS, tw, lane, bid);
    const T inv2mu0 = (T)S.inv2mu0, Bc = (T)S.Bc;
    const T sc = (T)(1.0 / ((double)NX * (double)ny));
    const int ky = ky0 + t;
    // the wave direction in the pass precision (FP32 phase: float)
    const T uy = (T)fftfreq(ky, ny) / (T)ny;
    const bool nqy = (ny & 1) == 0 && 2 * ky == ny;
    for (int kx = lane; kx < NX; kx += G) {
      const int pk = pidx<C>(kx);
      C* pxx = &l0[pk];
      C* pyy = &l0[LS + pk];
      C* pxy = &l0[2 * LS + pk];
      if (kx == 0 && ky == 0) {
        *pxx = mk<C>(T(0), T(0)); *pyy = *pxx; *pxy = *pxx;
        continue;
      }
      const T ux = (T)fftfreq(kx, NX) / (T)NX;
      const T inv = T(1) / sqrt(ux * ux + uy * uy);
      const T nxv = ux * inv, nyv = uy * inv;
      const C txx = *pxx, tyy = *pyy, txy = *pxy;
      C exx, eyy, exy;
      gamma2d_apply(txx, tyy, txy, nxv, nyv, inv2mu0, Bc, exx, eyy, exy);
      const bool nqx = 2 * kx == NX;
      if (nqx || nqy) {
        C fxx, fyy, fxy;
        gamma2d_apply(txx, tyy, txy, nqx ? -nxv : nxv, nqy ? -nyv : nyv, inv2mu0, Bc, fxx, fyy, fxy);
        exx = mk<C>(T(0.5) * (exx.x + fxx.x), T(0.5) * (exx.y + fxx.y));
        eyy = mk<C>(T(0.5) * (eyy.x + fyy.x), T(0.5) * (eyy.y + fyy.y));
        exy = mk<C>(T(0.5) * (exy.x + fxy.x), T(0.5) * (exy.y + fxy.y));
      }
      *pxx = mk<C>(exx.x * sc, exx.y * sc);
      *pyy = mk<C>(eyy.x * sc, eyy.y * sc);
      *pxy = mk<C>(exy.x * sc, exy.y * sc);
    }
    grp_sync<G>(bid);
    warp_fft<NX, +1, 1, G>(l0, LS, tw, lane, bid);
    warp_fft<NX, +1, 1, G>(l0 + LS, LS, tw, lane, bid);
    warp_fft<NX, +1, 1, G>(l0 + 2 * LS, LS, tw, lane, bid);
  }
  __syncthreads();
  for (int e = threadIdx.x; e < TOT; e += G * kColTiles) {
    const int c = e / (NX * kColTiles);
    const int rem = e - c * NX * kColTiles;
    const int x = rem / kColTiles, tt = rem - x * kColTiles;
    if (tt < tcw) spec[((size_t)c * NX + x) * ld + ky0 + tt] = lines[(c * kColTiles + tt) * PL + pidx<C>(x)];
  }
}

template <typename T, int MAXN>
__global__ void __launch_bounds__(col_threads(MAXN), MAXN <= 256 ? (sizeof(T) == 4 ? MGK_COL_MINB32 : 4) : 1) ls2d_col_fast_kernel(const Ls2dRep* __restrict__ reps,
                                                                       const Ls2dState* __restrict__ st,
                                                                       const int* __restrict__ col_map,
                                                                       const int* __restrict__ col_local) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int item = blockIdx.x;
  const int r = col_map[item];
  const Ls2dRep& R = reps[r];
  const Ls2dState& S = st[r];
  if (S.done != 0) return;
  const int ky0 = col_local[item] * fast_col_tiles(MAXN);
#define MGK_COL_CASE(n) \
  case n: if constexpr (n <= MAXN) col_fast_body<T, n, fast_col_tiles(MAXN), fast_group(MAXN)>(R, S, ky0, smem_raw); break;
  switch (R.nx) {
    MGK_COL_CASE(64) MGK_COL_CASE(96) MGK_COL_CASE(128) MGK_COL_CASE(192) MGK_COL_CASE(256) MGK_COL_CASE(384)
    MGK_COL_CASE(512) MGK_COL_CASE(768) MGK_COL_CASE(1024)
    default: break;
  }
#undef MGK_COL_CASE
}

// Mixed plans, between the phases: FP64 field from the FP32 one.
// grid = (G, nsel).
__global__ void ls2d_promote_kernel(const Ls2dRep* reps, const int* sel) {
  const int r = sel[blockIdx.y];
  const Ls2dRep& R = reps[r];
  const long long n3 = 3 * R.N;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n3;
       i += (long long)gridDim.x * blockDim.x)
    R.eps[i] = (double)R.eps32[i];
}

// Replicas that finished phase 1 re-enter for phase 2; resets the control block.
__global__ void ls2d_phase2_kernel(Ls2dState* st, const int* sel, int nsel, Ls2dCtl* ctl) {
  if (threadIdx.x != 0) return;
  unsigned int n = 0;
  for (int q = 0; q < nsel; ++q) {
    Ls2dState& S = st[sel[q]];
    if (S.done == 1) { S.done = 0; S.phase_iter = 0; ++n; }
  }
  ctl->n_active = n;
  ctl->decided = 0;
  ctl->still = 0;
  ctl->bodies = 0;
  ctl->any = n > 0;
}

// Outputs in the reference layout: eps, sig (nx,ny,2,2) and partial sums of
// their components for the means (linear_elastic_simulator.py:83-88).
// grid = (G, nsel).
template <int LAW = 0>  // 1: the secant law, 2: the Rose law, 3: the Landau law
__global__ void ls2d_output_kernel(const Ls2dRep* reps, const Ls2dState* st, const int* sel, double* partials) {
  __shared__ double red[32];
  const int r = sel[blockIdx.y];
  const Ls2dRep& R = reps[r];
  const Ls2dState& S = st[r];
  const long long N = R.N;
  const double abar = S.abar;
  double* eps_out = R.out_eps;
  double* sig_out = R.out_sig;
  const int law_ps = R.law_ps;
  const double law_a = R.law_a, law_b = R.law_b;
  const bool capped_mix = R.aa && S.done == 2 && S.status == MGK_NOT_CONVERGED;
  double gam[kAaMax];
  const int nmix = capped_mix ? aa_load(R, gam) : 0;
  double s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N;
       i += (long long)gridDim.x * blockDim.x) {
    double ev[3] = {R.eps[i], R.eps[N + i], R.eps[2 * N + i]};
    if (capped_mix) aa_mix_voxel(R, i, nmix, gam, ev);  // the loop ended at the cap: the last mixed iterate
    const double sxy = ev[2];
    const double exx = ev[0], eyy = ev[1];
    const double exy = abar == 0 ? sxy : sxy + abar;
    const double eyx = abar == 0 ? sxy : sxy - abar;
    double pxx = R.ep[i], pyy = R.ep[N + i], pxy, pyx;
    if (R.epa) { pxy = R.epa[i]; pyx = R.epa[N + i]; }
    else { pxy = R.ep[2 * N + i]; pyx = pxy; }
    const double lam = R.lam[i];
    const double dxx = exx - pxx, dxy = exy - pxy, dyx = eyx - pyx, dyy = eyy - pyy;
    double mu = R.mu[i];
    double sxx, syy, sxy2, syx2;
    if constexpr (LAW == 3) {
      landau_sigma(mu, lam, dxx, dyy, dxy, dyx, R.lp, law_ps, sxx, syy, sxy2, syx2, R.out_e33 ? R.out_e33 + i : nullptr);
    } else if constexpr (LAW == 2) {
      // Rose: sigma_yx is a copy of sigma_xy, from the [0,1] strain entry
      law_sigma<2>(mu, lam, dxx, dyy, dxy, law_a, law_b, law_ps, sxx, syy, sxy2);
      syx2 = sxy2;
    } else {
      if constexpr (LAW == 1) mu = secant_mu(mu, dxx, dyy, 0.5 * (dxy + dyx), law_a, law_b);
      const double tr = dxx + dyy;
      sxx = 2 * mu * dxx + lam * tr;
      syy = 2 * mu * dyy + lam * tr;
      sxy2 = 2 * mu * dxy;
      syx2 = 2 * mu * dyx;
    }
    if (eps_out) reinterpret_cast<double4*>(eps_out)[i] = make_double4(exx, exy, eyx, eyy);
    if (sig_out) reinterpret_cast<double4*>(sig_out)[i] = make_double4(sxx, sxy2, syx2, syy);
    s[0] += exx; s[1] += exy; s[2] += eyx; s[3] += eyy;
    s[4] += sxx; s[5] += sxy2; s[6] += syx2; s[7] += syy;
  }
  for (int q = 0; q < 8; ++q) {
    double t = block_sum(s[q], red);
    if (threadIdx.x == 0) partials[((size_t)blockIdx.y * gridDim.x + blockIdx.x) * 8 + q] = t;
  }
}

// Anderson mixing over fields of n doubles (linear_elastic_simulator.py:
// 1185-1209), kept as differences: hist holds 2 m + 2 vectors of n doubles,
// dF columns 0..m-1, dG columns 0..m-1, then f_prev and g_prev.  One pass
// forms f = g - x, writes column `slot` (dF = f - f_prev, dG = g - g_prev)
// when a previous pair exists, stores f and g as the previous pair, and
// accumulates <dF_j, dF_slot> and <dF_j, f> for the ncols valid columns.
constexpr int kAaBlocks = 296;

__global__ void __launch_bounds__(256) aa_update_kernel(long long n, const double* __restrict__ x,
                                                        const double* __restrict__ g, double* __restrict__ hist,
                                                        int m, int slot, int have_prev, int ncols,
                                                        double* __restrict__ partials) {
  __shared__ double red[32];
  double* dF = hist;
  double* dG = hist + (size_t)m * n;
  double* fp = hist + 2 * (size_t)m * n;
  double* gp = fp + n;
  double an[kAaMax], ar[kAaMax];
#pragma unroll
  for (int j = 0; j < kAaMax; ++j) { an[j] = 0.0; ar[j] = 0.0; }
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double gi = g[i], fi = gi - x[i];
    double df = 0.0;
    if (have_prev) {
      df = fi - fp[i];
      dF[(size_t)slot * n + i] = df;
      dG[(size_t)slot * n + i] = gi - gp[i];
    }
    fp[i] = fi;
    gp[i] = gi;
#pragma unroll
    for (int j = 0; j < kAaMax; ++j)
      if (j < ncols) {
        const double c = (j == slot && have_prev) ? df : dF[(size_t)j * n + i];
        an[j] += c * df;
        ar[j] += c * fi;
      }
  }
#pragma unroll
  for (int j = 0; j < kAaMax; ++j)
    if (j < ncols) {
      const double a = block_sum(an[j], red);
      const double b = block_sum(ar[j], red);
      if (threadIdx.x == 0) {
        partials[(size_t)blockIdx.x * 2 * kAaMax + j] = a;
        partials[(size_t)blockIdx.x * 2 * kAaMax + kAaMax + j] = b;
      }
    }
}

// sums the per-block partials: out[j] = <dF_j, dF_slot>, out[kAaMax + j] = <dF_j, f>
__global__ void aa_sum_kernel(const double* __restrict__ partials, int nb, int ncols, double* __restrict__ out) {
  __shared__ double red[32];
  for (int q = 0; q < 2 * kAaMax; ++q) {
    if ((q % kAaMax) >= ncols) continue;
    double a = 0.0;
    for (int b = threadIdx.x; b < nb; b += blockDim.x) a += partials[(size_t)b * 2 * kAaMax + q];
    a = block_sum(a, red);
    if (threadIdx.x == 0) out[q] = a;
  }
}

struct AaCoef { double v[kAaMax]; };

// x = g - sum_j gamma_j dG_j
__global__ void aa_mix_kernel(long long n, const double* __restrict__ g, const double* __restrict__ hist, int m,
                              int ncols, AaCoef gam, double* __restrict__ x) {
  const double* dG = hist + (size_t)m * n;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    double s = 0.0;
#pragma unroll
    for (int j = 0; j < kAaMax; ++j)
      if (j < ncols) s += gam.v[j] * dG[(size_t)j * n + i];
    x[i] = g[i] - s;
  }
}


// ------------------------------------- Anderson mixing inside the LS loop ---
// Type-II Anderson mixing of one replica's fixed-point iterates, run in the
// loop body between the row kernel that forms the image g = G(x) (with the
// update norm and the convergence decision) and the first row pass of the
// next iterate (linear_elastic_simulator.py:1185-1209): residual f = g - x;
// differences dF, dG of consecutive (f, g) pairs, at most m of them;
// gamma = argmin |dF gamma - f|; x = g - dG gamma.  When the coefficients are
// not finite the step is the plain one (x = g) and the history restarts from
// the last pair, as the reference's fallback does.  Fields are the replica's
// symmetric strain planes (xx, yy, xy); inner products weight the xy plane
// by 2, as the reference's sums over the four tensor entries do.  The
// differences sit in a ring of m slots; the least-squares solution does not
// depend on the order of the columns.

// Mixing follows every iteration except the converged or non-finite one:
// the reference leaves its loop with the image g there, and with the last
// mixed iterate when the iteration cap ends the loop.
__device__ __forceinline__ bool aa_skip(const Ls2dState& S) {
  return S.done != 0 && S.status != MGK_NOT_CONVERGED;
}

// Ring buffer of one plan (n3 = 3 N doubles each): x, f_prev, g_prev, then
// dF slots 0 .. m-1 and dG slots 0 .. m-1.
__global__ void ls2d_aa_init_kernel(const Ls2dRep* reps, const int* sel, double* buf, Ls2dAA* aa) {
  const Ls2dRep& R = reps[sel[0]];
  const long long n3 = 3 * R.N;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n3; i += (long long)gridDim.x * blockDim.x)
    buf[i] = R.eps[i];
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    aa->k = 0;
    aa->slot_next = 0;
    aa->have_prev = 0;
    aa->nmix = 0;
    aa->ctr = 0;
  }
}

// Sum over the warp, the same value in every lane (reduced to lane 0, then
// broadcast: a butterfly would round differently per lane).
__device__ __forceinline__ double warp_allsum(double v) {
  return __shfl_sync(0xffffffffu, warp_sum(v), 0);
}

// Least squares of the mix, one warp (lanes = matrix rows): gamma = sum
// over eigenpairs (lambda_i, v_i) of the k x k Gram matrix with lambda_i
// above 1e-14 lambda_max of (v_i . b / lambda_i) v_i, the minimum-norm
// solution with the small singular values of dF cut off.  Eigenpairs by
// cyclic Jacobi rotations (Golub & Van Loan, Matrix Computations, 8.5), each
// rotation's row and column updates spread over the lanes.  sa, sv: k x k
// shared scratch; b in sb.  Writes gamma and nmix (0 for the plain step,
// and the history restarts from the last pair when the coefficients are
// not finite).
// Fast path of the same least squares (one thread): when the Gram matrix
// is comfortably conditioned no eigenvalue falls under the cut-off, so the
// truncated eigen solution is A^-1 b, solved here by Cholesky.  The test:
// lambda_min >= 1 / tr(A^-1) = 1 / ||L^-1||_F^2 and lambda_max <= tr(A);
// when 1 / ||L^-1||_F^2 > 1e-12 tr(A) every eigenvalue is above
// 1e-14 lambda_max with margin for the rounding of the estimate.  Returns
// false (nothing written) when the factorisation fails or the test does not
// hold: the eigen path decides then.
__device__ bool aa_lstsq_cholesky(Ls2dAA* aa, int k, const double* sb) {
  double Lm[kAaMax][kAaMax];
  double tr = 0.0;
  for (int i = 0; i < k; ++i) tr += aa->A[i][i];
  for (int j = 0; j < k; ++j) {
    double d = aa->A[j][j];
    for (int q = 0; q < j; ++q) d -= Lm[j][q] * Lm[j][q];
    if (!(d > 0.0)) return false;
    const double ljj = sqrt(d);
    Lm[j][j] = ljj;
    for (int i = j + 1; i < k; ++i) {
      double v = aa->A[i][j];
      for (int q = 0; q < j; ++q) v -= Lm[i][q] * Lm[j][q];
      Lm[i][j] = v / ljj;
    }
  }
  // ||L^-1||_F^2, column by column of L^-1 (forward substitution on e_c)
  double fro = 0.0;
  for (int c = 0; c < k; ++c) {
    double z[kAaMax];
    for (int i = 0; i < k; ++i) {
      double v = i == c ? 1.0 : 0.0;
      for (int q = c; q < i; ++q) v -= Lm[i][q] * z[q];
      z[i] = i < c ? 0.0 : v / Lm[i][i];
      if (i >= c) fro += z[i] * z[i];
    }
  }
  if (!(isfinite(fro) && 1.0 / fro > 1e-12 * tr)) return false;
  double y[kAaMax], g[kAaMax];
  for (int i = 0; i < k; ++i) {
    double v = sb[i];
    for (int q = 0; q < i; ++q) v -= Lm[i][q] * y[q];
    y[i] = v / Lm[i][i];
  }
  for (int i = k - 1; i >= 0; --i) {
    double v = y[i];
    for (int q = i + 1; q < k; ++q) v -= Lm[q][i] * g[q];
    g[i] = v / Lm[i][i];
  }
  for (int i = 0; i < k; ++i)
    if (!isfinite(g[i])) return false;
  for (int i = 0; i < k; ++i) aa->gamma[i] = g[i];
  aa->nmix = k;
  return true;
}

__device__ void aa_lstsq_warp(Ls2dAA* aa, int k, double (*sa)[kAaMax], double (*sv)[kAaMax], const double* sb) {
  const int l = threadIdx.x;  // lane, < 32
  for (int e = l; e < k * k; e += 32) {
    const int i = e / k, j = e - (e / k) * k;
    sa[i][j] = aa->A[i][j];
    sv[i][j] = i == j ? 1.0 : 0.0;
  }
  __syncwarp();
  double fro = 0.0;
  for (int e = l; e < k * k; e += 32) {
    const int i = e / k, j = e - (e / k) * k;
    fro += sa[i][j] * sa[i][j];
  }
  fro = warp_allsum(fro);
  for (int sweep = 0; sweep < 40; ++sweep) {
    double off = 0.0;
    for (int e = l; e < k * k; e += 32) {
      const int i = e / k, j = e - (e / k) * k;
      if (j > i) off += sa[i][j] * sa[i][j];
    }
    off = warp_allsum(off);
    if (!(off > 1e-30 * fro)) break;  // also leaves on NaN (uniform: every lane has the same sums)
    for (int p = 0; p < k; ++p)
      for (int q = p + 1; q < k; ++q) {
        const double apq = sa[p][q], app = sa[p][p], aqq = sa[q][q];
        __syncwarp();
        if (fabs(apq) <= 1e-18 * sqrt(fabs(app * aqq))) {  // negligible: no rotation
          if (l == 0) { sa[p][q] = 0.0; sa[q][p] = 0.0; }
          __syncwarp();
          continue;
        }
        const double th = (aqq - app) / (2.0 * apq);
        const double t = (th >= 0.0 ? 1.0 : -1.0) / (fabs(th) + sqrt(th * th + 1.0));
        const double c = 1.0 / sqrt(t * t + 1.0), sn = t * c;
        double x0 = 0.0, x1 = 0.0;
        if (l < k) { x0 = sa[l][p]; x1 = sa[l][q]; }
        __syncwarp();
        if (l < k) { sa[l][p] = c * x0 - sn * x1; sa[l][q] = sn * x0 + c * x1; }
        __syncwarp();
        if (l < k) { x0 = sa[p][l]; x1 = sa[q][l]; }
        __syncwarp();
        if (l < k) {
          sa[p][l] = c * x0 - sn * x1;
          sa[q][l] = sn * x0 + c * x1;
          const double v0 = sv[l][p], v1 = sv[l][q];
          sv[l][p] = c * v0 - sn * v1;
          sv[l][q] = sn * v0 + c * v1;
        }
        __syncwarp();
      }
  }
  double lmax = 0.0;
  for (int i = 0; i < k; ++i) lmax = fmax(lmax, sa[i][i]);
  // gamma_j (lane j) = sum_i [lambda_i kept] v_ji (v_i . b) / lambda_i
  double g = 0.0;
  bool ok = isfinite(lmax);
  if (ok && lmax > 0.0 && l < k) {
    for (int i = 0; i < k; ++i) {
      const double li = sa[i][i];
      if (!(li > 1e-14 * lmax)) continue;
      double vb = 0.0;
      for (int j = 0; j < k; ++j) vb += sv[j][i] * sb[j];
      g += sv[l][i] * (vb / li);
    }
  }
  ok = __all_sync(0xffffffffu, ok && (l >= k || isfinite(g)));
  if (!ok) {  // the plain step; the history restarts from the last pair
    if (l == 0) {
      aa->k = 0;
      aa->slot_next = 0;
      aa->nmix = 0;
    }
    return;
  }
  if (l < k) aa->gamma[l] = g;
  if (l == 0) aa->nmix = k;
}

// f = g - x; with a previous pair, the new column dF = f - f_prev and
// dG = g - g_prev goes to slot slot_next; (f, g) become the previous pair.
// Per-block partial sums of <dF_j, dF_new> and <dF_j, f> over the columns
// valid after this update; the last block to finish sums them, updates the
// Gram matrix and solves the least-squares problem of the mix.
constexpr int kAaThreads = 256, kAaWarps = kAaThreads / 32;
// K: the history depth m, compile-time so that only m accumulator pairs
// live in registers
template <int K>
__global__ void __launch_bounds__(kAaThreads) ls2d_aa_update_kernel(const Ls2dRep* reps, const Ls2dState* st,
                                                                    const int* sel, double* buf, Ls2dAA* aa, int m,
                                                                    double* part) {
  __shared__ double wred[kAaWarps][2 * kAaMax];
  __shared__ double lred[kAaThreads / (2 * kAaMax)][2 * kAaMax];
  __shared__ double sums[2 * kAaMax];
  __shared__ double sa[kAaMax][kAaMax], sv[kAaMax][kAaMax];
  __shared__ int s_last;
  const int r = sel[0];
  const Ls2dRep& R = reps[r];
  if (aa_skip(st[r])) return;
  const long long N = R.N, n3 = 3 * N;
  const int have_prev = aa->have_prev;
  const int slot = have_prev ? aa->slot_next : -1;
  const int ncols = have_prev ? min(aa->k + 1, m) : aa->k;
  const double* x = buf;
  double* fp = buf + n3;
  double* gp = buf + 2 * n3;
  double* dF = buf + 3 * n3;
  double* dG = dF + (size_t)m * n3;
  double an[K], ar[K];
#pragma unroll
  for (int j = 0; j < K; ++j) { an[j] = 0.0; ar[j] = 0.0; }
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n3; i += (long long)gridDim.x * blockDim.x) {
    const double w = i >= 2 * N ? 2.0 : 1.0;
    const double gi = R.eps[i], fi = gi - x[i];
    double df = 0.0;
    if (have_prev) {
      df = fi - fp[i];
      dF[(size_t)slot * n3 + i] = df;
      dG[(size_t)slot * n3 + i] = gi - gp[i];
    }
    fp[i] = fi;
    gp[i] = gi;
#pragma unroll
    for (int j = 0; j < K; ++j)
      if (j < ncols) {
        const double c = w * (j == slot ? df : dF[(size_t)j * n3 + i]);
        an[j] += c * df;
        ar[j] += c * fi;
      }
  }
  // block partials in a fixed order: warp trees, then the warps in order
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int j = 0; j < K; ++j)
    if (j < ncols) {
      const double a = warp_sum(an[j]), b = warp_sum(ar[j]);
      if (lane == 0) { wred[wid][j] = a; wred[wid][kAaMax + j] = b; }
    }
  __syncthreads();
  constexpr int Q = 2 * kAaMax;
  if (threadIdx.x < Q && threadIdx.x % kAaMax < ncols) {
    double t = 0.0;
    for (int w = 0; w < kAaWarps; ++w) t += wred[w][threadIdx.x];
    part[(size_t)blockIdx.x * Q + threadIdx.x] = t;
    __threadfence();
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned int t = atomicInc(&aa->ctr, gridDim.x - 1);  // self-resetting
    s_last = t == gridDim.x - 1;
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  // the last block: sums over the blocks (value q = thread % Q, blocks in
  // strides of the thread's group, then the groups in order)
  const int nb = gridDim.x;
  {
    const int q = threadIdx.x % Q, g0 = threadIdx.x / Q;
    double a = 0.0;
    if (q % kAaMax < ncols)
      for (int b = g0; b < nb; b += kAaThreads / Q) a += __ldcg(&part[(size_t)b * Q + q]);
    lred[g0][q] = a;
  }
  __syncthreads();
  if (threadIdx.x < Q) {
    double t = 0.0;
    for (int g = 0; g < kAaThreads / Q; ++g) t += lred[g][threadIdx.x];
    sums[threadIdx.x] = t;
  }
  __syncthreads();
  if (threadIdx.x >= 32) return;
  if (threadIdx.x == 0) {
    if (have_prev) {
      for (int j = 0; j < ncols; ++j) {
        aa->A[slot][j] = sums[j];
        aa->A[j][slot] = sums[j];
      }
      aa->k = ncols;
      aa->slot_next = (slot + 1) % m;
    }
    aa->have_prev = 1;
    aa->nmix = 0;
  }
  __syncwarp();
  if (ncols == 0) return;
  int fast = 0;
  if (threadIdx.x == 0) fast = aa_lstsq_cholesky(aa, ncols, sums + kAaMax) ? 1 : 0;
  if (__shfl_sync(0xffffffffu, fast, 0)) return;
  aa_lstsq_warp(aa, ncols, sa, sv, sums + kAaMax);
}


}  // namespace mgk

// ================================================================== plan ===
using namespace mgk;

namespace {

constexpr int kThreads = 256;
constexpr int kPerVoxelBlocks = 256;  // G: CTAs per replica for per-voxel kernels

int grid_blocks(long long maxN) {
  long long b = (maxN + kThreads - 1) / kThreads;
  if (b > kPerVoxelBlocks) b = kPerVoxelBlocks;
  if (b < 1) b = 1;
  return (int)b;
}

// columns per CTA: largest power of two <= 8 whose double-buffered tile fits
// `cap` bytes (keeps several CTAs resident per SM)
int pick_tc(int nx, size_t csz, size_t cap) {
  int tc = 8;
  while (tc > 1 && 2 * 3 * (size_t)tc * nx * csz > cap) tc >>= 1;
  return tc;
}

}  // namespace

struct mgk_ls2d_plan {
  int nrep = 0;
  int plane_mode = 0, prec = 0;
  long long maxN = 0;
  size_t row_smem = 0, col_smem = 0;      // FP64 iteration kernels
  size_t row_smem32 = 0, col_smem32 = 0;  // FP32 iteration kernels
  int fast = 0;                           // kernel family in use: 0 CTA-wide passes, 256/512/1024 warp-line
  int fast_nat = 0;                       // smallest warp-line family that covers every side (0: none)
  int law = 0;                            // 1: secant degradation law, 2: Rose law
  double law_a = 0, law_b = 0;            // the law's parameters (set_secant, set_rose)
  int law_ps = 0;
  std::vector<int> tc_gen;                // column tiles of the CTA-wide family, per replica
  std::vector<Ls2dRep> reps;      // host copy (static part)
  std::vector<char> has_material;
  Ls2dRep* h_reps = nullptr;      // pinned staging of the table
  int* h_maps = nullptr;          // pinned staging: row_map, row_local, col_map, col_local, sel
  Ls2dCtl* h_ctl = nullptr;
  Ls2dState* h_state = nullptr;
  cudaEvent_t staged = nullptr;   // last upload from the staging buffers
  bool staged_pending = false;
  Ls2dRep* d_reps = nullptr;
  Ls2dState* d_st = nullptr;
  Ls2dCtl* d_ctl = nullptr;
  int* d_maps = nullptr;
  unsigned int* d_repctr = nullptr;
  double* d_part = nullptr;
  double* d_mat_part = nullptr;   // partials of the material kernel
  size_t part_doubles = 0;
  int total_row_items = 0, total_col_items = 0;
  std::vector<void*> allocations;
  // spectra of all replicas, one slab
  void* spec_slab = nullptr;
  size_t spec_bytes = 0;
  // loop graph for the current selection
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int graph_mode = -1;  // -1 untried, 1 while-node graph, 0 host loop
  int graph_cap = 0;
  int graph_aa = 0;     // Anderson depth of the current graph
  // instantiated loop graphs by selection shape (a serving loop selects
  // varying numbers of replicas; each shape is built once)
  struct GraphEntry {
    int rows, cols, nsel, cap, aa;
    cudaGraph_t g;
    cudaGraphExec_t x;
  };
  std::vector<GraphEntry> gcache;
  // selection of the last call
  int nsel = 0, sel_rows = 0, sel_cols = 0;
  // persistent bulk-prefetch row kernels (0 when a replica has odd ny or the
  // stages do not fit): stage bytes, dynamic smem and resident CTAs per SM
  int tma = 0;
  int stage64 = 0, stage32 = 0;
  size_t tma_smem64 = 0, tma_smem32 = 0;
  int occ64 = 0, occ32 = 0, num_sms = 0;
  // Anderson mixing inside the loop (one replica per solve): depth, ring
  // buffer of (3 + 2 m) strain fields, state and per-block partial sums
  int aa_m = 0;
  double* aa_buf = nullptr;
  size_t aa_doubles = 0;
  Ls2dAA* d_aa = nullptr;
  double* aa_part = nullptr;
  int aa_nb = 0;
};

static int plan_alloc(mgk_ls2d_t p, void** ptr, size_t bytes) {
  if (cudaMalloc(ptr, bytes) != cudaSuccess) {
    cudaGetLastError();
    set_error("mgk_ls2d: cudaMalloc of %zu bytes failed", bytes);
    return MGK_OOM;
  }
  p->allocations.push_back(*ptr);
  return MGK_OK;
}

// warp-line kernel variants: sides up to 256, or up to 512 (more registers)
template <typename TS, bool IN_SPEC, bool FINAL>
static void* row_fast_fn(int fast, int law = 0) {
  if constexpr (sizeof(TS) == 8) {
    if (law == 1)  // the secant law (FP64 plans only)
      return fast > 512   ? (void*)ls2d_row_fast_kernel<TS, 1024, IN_SPEC, FINAL, 1>
             : fast > 256 ? (void*)ls2d_row_fast_kernel<TS, 512, IN_SPEC, FINAL, 1>
                          : (void*)ls2d_row_fast_kernel<TS, 256, IN_SPEC, FINAL, 1>;
    if (law == 2)  // the Rose law (FP64 plans only)
      return fast > 512   ? (void*)ls2d_row_fast_kernel<TS, 1024, IN_SPEC, FINAL, 2>
             : fast > 256 ? (void*)ls2d_row_fast_kernel<TS, 512, IN_SPEC, FINAL, 2>
                          : (void*)ls2d_row_fast_kernel<TS, 256, IN_SPEC, FINAL, 2>;
    if (law == 3)  // the Landau law (FP64 plans only)
      return fast > 512   ? (void*)ls2d_row_fast_kernel<TS, 1024, IN_SPEC, FINAL, 3>
             : fast > 256 ? (void*)ls2d_row_fast_kernel<TS, 512, IN_SPEC, FINAL, 3>
                          : (void*)ls2d_row_fast_kernel<TS, 256, IN_SPEC, FINAL, 3>;
  }
  return fast > 512   ? (void*)ls2d_row_fast_kernel<TS, 1024, IN_SPEC, FINAL>
         : fast > 256 ? (void*)ls2d_row_fast_kernel<TS, 512, IN_SPEC, FINAL>
                      : (void*)ls2d_row_fast_kernel<TS, 256, IN_SPEC, FINAL>;
}
template <typename TS>
static void* col_fast_fn(int fast) {
  return fast > 512   ? (void*)ls2d_col_fast_kernel<TS, 1024>
         : fast > 256 ? (void*)ls2d_col_fast_kernel<TS, 512>
                      : (void*)ls2d_col_fast_kernel<TS, 256>;
}

template <typename T>
static int ls2d_set_fast_attrs(int fast, size_t row_smem, size_t col_smem) {
  void* fns[16] = {row_fast_fn<T, true, true>(fast), row_fast_fn<T, false, true>(fast),
                   row_fast_fn<T, true, false>(fast), row_fast_fn<T, false, false>(fast),
                   row_fast_fn<T, true, true>(fast, 1), row_fast_fn<T, false, true>(fast, 1),
                   row_fast_fn<T, true, false>(fast, 1), row_fast_fn<T, false, false>(fast, 1),
                   row_fast_fn<T, true, true>(fast, 2), row_fast_fn<T, false, true>(fast, 2),
                   row_fast_fn<T, true, false>(fast, 2), row_fast_fn<T, false, false>(fast, 2),
                   row_fast_fn<T, true, true>(fast, 3), row_fast_fn<T, false, true>(fast, 3),
                   row_fast_fn<T, true, false>(fast, 3), row_fast_fn<T, false, false>(fast, 3)};
  for (void* f : fns) MGK_CUDA(raise_smem((const void*)f, (int)row_smem));
  MGK_CUDA(raise_smem((const void*)col_fast_fn<T>(fast), (int)col_smem));
  return MGK_OK;
}

template <typename TS, typename TC>
static int ls2d_set_attrs(size_t row_smem, size_t col_smem) {
  MGK_CUDA(raise_smem((const void*)ls2d_row_kernel<TS, TC, true, true>, (int)row_smem));
  MGK_CUDA(raise_smem((const void*)ls2d_row_kernel<TS, TC, false, true>, (int)row_smem));
  MGK_CUDA(raise_smem((const void*)ls2d_row_kernel<TS, TC, true, false>, (int)row_smem));
  MGK_CUDA(raise_smem((const void*)ls2d_row_kernel<TS, TC, false, false>, (int)row_smem));
  MGK_CUDA(raise_smem((const void*)ls2d_col_kernel<TS, TC>, (int)col_smem));
  return MGK_OK;
}

extern "C" int mgk_ls2d_destroy(mgk_ls2d_t p) {
  if (!p) return MGK_OK;
  for (auto& e : p->gcache) {
    cudaGraphExecDestroy(e.x);
    cudaGraphDestroy(e.g);
  }
  if (p->staged) cudaEventDestroy(p->staged);
  for (void* a : p->allocations) cudaFree(a);
  if (p->aa_buf) cudaFree(p->aa_buf);
  if (p->d_aa) cudaFree(p->d_aa);
  if (p->aa_part) cudaFree(p->aa_part);
  if (p->h_reps) cudaFreeHost(p->h_reps);
  if (p->h_maps) cudaFreeHost(p->h_maps);
  if (p->h_ctl) cudaFreeHost(p->h_ctl);
  if (p->h_state) cudaFreeHost(p->h_state);
  delete p;
  return MGK_OK;
}

extern "C" int mgk_ls2d_create_batch(int nrep, const int* nxs, const int* nys, int plane_mode, int precision,
                                     mgk_ls2d_t* out) {
  MGK_REQUIRE(out != nullptr, "mgk_ls2d_create_batch: null output handle");
  *out = nullptr;
  MGK_REQUIRE(nrep >= 1 && nrep <= 65535 && nxs && nys, "mgk_ls2d_create_batch: bad replica count");
  MGK_REQUIRE(plane_mode == MGK_PLANE_STRAIN || plane_mode == MGK_PLANE_STRESS,
              "mgk_ls2d_create: plane_mode must be 0 (strain) or 1 (stress)");
  MGK_REQUIRE(precision == MGK_FP64 || precision == MGK_MIXED, "mgk_ls2d_create: bad precision");
  for (int r = 0; r < nrep; ++r) {
    FftLen f;
    MGK_REQUIRE(fft_schedule(nxs[r], &f) && fft_schedule(nys[r], &f) && nxs[r] % 2 == 0,
                "mgk_ls2d_create: grid %dx%d unsupported (each side 2^a 3^b up to 4096, nx even)", nxs[r],
                nys[r]);
    MGK_REQUIRE(2 * 3 * (size_t)nys[r] * sizeof(double2) <= 220 * 1024 &&
                    2 * 3 * (size_t)pick_tc(nxs[r], sizeof(double2), 64 * 1024) * nxs[r] * sizeof(double2) <=
                        220 * 1024,
                "mgk_ls2d_create: grid too large for the shared-memory FFT");
  }
  mgk_ls2d_t p = new mgk_ls2d_plan();
  p->nrep = nrep;
  p->plane_mode = plane_mode;
  p->prec = precision;
  const bool mixed = precision == MGK_MIXED;
  const size_t c64 = sizeof(double2);
  auto fail = [&](int s) { mgk_ls2d_destroy(p); return s; };
  p->reps.resize(nrep);
  p->has_material.assign(nrep, 0);
  {
    bool fast = true;
    int side = 0;
    for (int r = 0; r < nrep; ++r) {
      fast = fast && warp_fft_len(nxs[r]) && warp_fft_len(nys[r]);
      side = std::max(side, std::max(nxs[r], nys[r]));
    }
    p->fast_nat = fast ? (side > 512 ? 1024 : side > 256 ? 512 : 256) : 0;
    const char* env = getenv("MGK_FAST");
    p->fast = (env && env[0] == '0') ? 0 : p->fast_nat;
  }
  p->tc_gen.resize(nrep);
  std::vector<size_t> spec_off(nrep, 0);
  int total_col_max = 0;
  size_t row_smem = 0, col_smem = 0, row_smem32 = 0, col_smem32 = 0;
  for (int r = 0; r < nrep; ++r) {
    const int nx = nxs[r], ny = nys[r];
    Ls2dRep& R = p->reps[r];
    memset(&R, 0, sizeof(R));
    R.nx = nx; R.ny = ny; R.nyh = ny / 2 + 1; R.ld = R.nyh;
    R.N = (long long)nx * ny;
    p->tc_gen[r] = pick_tc(nx, c64, 64 * 1024);
    R.tc = p->fast ? fast_col_tiles(p->fast) : p->tc_gen[r];
    R.row_items = nx / 2;
    R.col_items = (R.nyh + R.tc - 1) / R.tc;
    {
      int cmax = (R.nyh + p->tc_gen[r] - 1) / p->tc_gen[r];
      for (int v : {256, 512, 1024})
        if (p->fast_nat && v >= p->fast_nat) cmax = std::max(cmax, (R.nyh + fast_col_tiles(v) - 1) / fast_col_tiles(v));
      total_col_max += cmax;
    }
    fft_schedule(nx, &R.fx64);
    fft_schedule(ny, &R.fy64);
    R.fx32 = R.fx64;
    R.fy32 = R.fy64;
    R.fx64.tw = twiddles(nx, MGK_FP64);
    R.fy64.tw = twiddles(ny, MGK_FP64);
    if (!R.fx64.tw || !R.fy64.tw) return fail(MGK_OOM);
    if (mixed) {
      R.fx32.tw = twiddles(nx, 1 /* float table */);
      R.fy32.tw = twiddles(ny, 1 /* float table */);
      if (!R.fx32.tw || !R.fy32.tw) return fail(MGK_OOM);
    }
    if (p->fast) {
      row_smem = std::max(row_smem, (size_t)row_fast_smem(ny, 16, 8));
      col_smem = std::max(col_smem, (size_t)col_fast_smem(nx, 16, R.tc));
      row_smem32 = std::max(row_smem32, (size_t)row_fast_smem(ny, 8, 4));
      col_smem32 = std::max(col_smem32, (size_t)col_fast_smem(nx, 8, R.tc));
    } else {
      row_smem = std::max(row_smem, 2 * 3 * (size_t)ny * c64);
      col_smem = std::max(col_smem, 2 * 3 * (size_t)R.tc * nx * c64);
      row_smem32 = row_smem / 2;
      col_smem32 = col_smem / 2;
    }
    p->maxN = std::max(p->maxN, R.N);
    p->total_row_items += R.row_items;
    p->total_col_items += R.col_items;
    void* f = nullptr;
    int st = plan_alloc(p, &f, sizeof(double) * R.N * 10);
    if (st) return fail(st);
    double* d = reinterpret_cast<double*>(f);
    R.mu = d; R.lam = d + R.N; R.eps = d + 2 * R.N; R.ep = d + 5 * R.N; R.epa = nullptr;
    // spectra of all replicas sit in one slab (assigned after the loop)
    spec_off[r] = p->spec_bytes;
    p->spec_bytes += (3 * (size_t)nx * R.ld * c64 + 255) / 256 * 256;
    if (mixed) {
      void* g = nullptr;
      st = plan_alloc(p, &g, sizeof(float) * R.N * 8);
      if (st) return fail(st);
      float* fl = reinterpret_cast<float*>(g);
      R.mu32 = fl; R.lam32 = fl + R.N; R.eps32 = fl + 2 * R.N; R.ep32 = fl + 5 * R.N;
    }
  }
  {
    void* slab = nullptr;
    int st = plan_alloc(p, &slab, p->spec_bytes);
    if (st) return fail(st);
    p->spec_slab = slab;
    for (int r = 0; r < nrep; ++r) p->reps[r].spec = reinterpret_cast<char*>(slab) + spec_off[r];
  }
  p->row_smem = row_smem;
  p->col_smem = col_smem;
  p->row_smem32 = row_smem32;
  p->col_smem32 = col_smem32;
  int st = p->fast ? ls2d_set_fast_attrs<double>(p->fast, row_smem, col_smem) : ls2d_set_attrs<double, double>(row_smem, col_smem);
  if (st == MGK_OK && mixed)
    st = p->fast ? ls2d_set_fast_attrs<float>(p->fast, row_smem32, col_smem32) : ls2d_set_attrs<float, float>(row_smem32, col_smem32);
  if (st) return fail(st);
  {
    // persistent bulk-prefetch row kernels: every replica needs ny even
    bool ok = true;
    int st64 = 0, st32 = 0, maxny = 0;
    for (const Ls2dRep& R : p->reps) {
      ok = ok && (R.ny % 2 == 0);
      st64 = std::max(st64, (int)(6 * R.ld * sizeof(double2) + 16 * R.ny * sizeof(double)));
      st32 = std::max(st32, (int)(6 * R.ld * sizeof(float2) + 16 * R.ny * sizeof(float)));
      maxny = std::max(maxny, R.ny);
    }
    st64 = (st64 + 127) / 128 * 128;
    st32 = (st32 + 127) / 128 * 128;
    const size_t sm64 = 2 * (size_t)st64 + 3 * (size_t)maxny * sizeof(double2);
    const size_t sm32 = 2 * (size_t)st32 + 3 * (size_t)maxny * sizeof(float2);
    // opt-in: at 256-point lines the per-CTA FFT work, not load latency,
    // bounds the row kernel, and the prefetching variant needs one CTA per SM
    const char* env = getenv("MGK_TMA");
    ok = ok && !p->fast && (env && env[0] == '1') && sm64 <= 220 * 1024;
    int dev = 0;
    if (ok && cudaGetDevice(&dev) == cudaSuccess &&
        cudaDeviceGetAttribute(&p->num_sms, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess) {
      p->stage64 = st64; p->stage32 = st32; p->tma_smem64 = sm64; p->tma_smem32 = sm32;
      bool good = raise_smem((const void*)ls2d_row_tma_kernel<double, double, true>, (int)sm64) == cudaSuccess &&
                  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&p->occ64, ls2d_row_tma_kernel<double, double, true>,
                                                                kThreads, sm64) == cudaSuccess;
      if (good && mixed)
        good = raise_smem((const void*)ls2d_row_tma_kernel<float, float, false>, (int)sm32) == cudaSuccess &&
               raise_smem((const void*)ls2d_row_tma_kernel<float, float, true>, (int)sm32) == cudaSuccess &&
               cudaOccupancyMaxActiveBlocksPerMultiprocessor(&p->occ32, ls2d_row_tma_kernel<float, float, false>,
                                                             kThreads, sm32) == cudaSuccess;
      p->tma = good && p->occ64 > 0 && (!mixed || p->occ32 > 0);
    }
    cudaGetLastError();
  }
  const int G = grid_blocks(p->maxN);
  p->part_doubles = std::max((size_t)2 * p->total_row_items, (size_t)nrep * G * 8);
  void* v = nullptr;
  if ((st = plan_alloc(p, &v, sizeof(double) * p->part_doubles))) return fail(st);
  p->d_part = reinterpret_cast<double*>(v);
  if ((st = plan_alloc(p, &v, sizeof(double) * 2 * kPerVoxelBlocks))) return fail(st);
  p->d_mat_part = reinterpret_cast<double*>(v);
  if ((st = plan_alloc(p, &v, sizeof(Ls2dRep) * nrep))) return fail(st);
  p->d_reps = reinterpret_cast<Ls2dRep*>(v);
  if ((st = plan_alloc(p, &v, sizeof(Ls2dState) * nrep))) return fail(st);
  p->d_st = reinterpret_cast<Ls2dState*>(v);
  if ((st = plan_alloc(p, &v, sizeof(Ls2dCtl)))) return fail(st);
  p->d_ctl = reinterpret_cast<Ls2dCtl*>(v);
  const size_t nmaps = 2 * (size_t)p->total_row_items + 2 * (size_t)std::max(p->total_col_items, total_col_max) + nrep;
  if ((st = plan_alloc(p, &v, sizeof(int) * nmaps))) return fail(st);
  p->d_maps = reinterpret_cast<int*>(v);
  if ((st = plan_alloc(p, &v, sizeof(unsigned int) * nrep))) return fail(st);
  p->d_repctr = reinterpret_cast<unsigned int*>(v);
  if (cudaMemset(p->d_repctr, 0, sizeof(unsigned int) * nrep) != cudaSuccess ||
      cudaMemset(p->d_st, 0, sizeof(Ls2dState) * nrep) != cudaSuccess ||
      cudaMemset(p->d_ctl, 0, sizeof(Ls2dCtl)) != cudaSuccess)
    return fail(MGK_CUDA_ERROR);
  if (cudaMallocHost(&p->h_reps, sizeof(Ls2dRep) * nrep) != cudaSuccess ||
      cudaMallocHost(&p->h_maps, sizeof(int) * nmaps) != cudaSuccess ||
      cudaMallocHost(&p->h_ctl, sizeof(Ls2dCtl)) != cudaSuccess ||
      cudaMallocHost(&p->h_state, sizeof(Ls2dState) * nrep) != cudaSuccess)
    return fail(MGK_OOM);
  if (cudaEventCreateWithFlags(&p->staged, cudaEventDisableTiming) != cudaSuccess) return fail(MGK_CUDA_ERROR);
  memcpy(p->h_reps, p->reps.data(), sizeof(Ls2dRep) * nrep);
  if (cudaMemcpy(p->d_reps, p->h_reps, sizeof(Ls2dRep) * nrep, cudaMemcpyHostToDevice) != cudaSuccess)
    return fail(MGK_CUDA_ERROR);
  *out = p;
  return MGK_OK;
}

extern "C" int mgk_ls2d_create(int nx, int ny, int plane_mode, int precision, mgk_ls2d_t* out) {
  return mgk_ls2d_create_batch(1, &nx, &ny, plane_mode, precision, out);
}

// wait until the previous upload from the pinned staging buffers has run
static int staging_wait(mgk_ls2d_t p) {
  if (p->staged_pending) {
    MGK_CUDA(cudaEventSynchronize(p->staged));
    p->staged_pending = false;
  }
  return MGK_OK;
}

static int ls2d_set_fields(mgk_ls2d_t p, int rep, const double* E, const double* nu, const double* epsp,
                           int set_moduli, cudaStream_t s) {
  Ls2dRep& R = p->reps[rep];
  const bool want_epa = epsp != nullptr;
  if (want_epa != (R.epa != nullptr)) {
    R.epa = want_epa ? R.mu + 8 * R.N : nullptr;
    int st = staging_wait(p);
    if (st) return st;
    p->h_reps[rep] = R;
    MGK_CUDA(cudaMemcpyAsync(&p->d_reps[rep], &p->h_reps[rep], sizeof(Ls2dRep), cudaMemcpyHostToDevice, s));
    MGK_CUDA(cudaEventRecord(p->staged, s));
    p->staged_pending = true;
  }
  const int grid = grid_blocks(R.N);
  ls2d_material_kernel<<<grid, kThreads, 0, s>>>(p->d_reps, rep, E, nu, epsp, p->plane_mode, set_moduli,
                                                 p->d_mat_part);
  MGK_CUDA(cudaGetLastError());
  if (set_moduli) {
    ls2d_medium_kernel<<<1, kThreads, 0, s>>>(p->d_reps, p->d_st, rep, p->d_mat_part, grid, p->plane_mode,
                                              set_moduli == 2 ? (p->law == 2 ? 2 : 1) : 0, p->law_b);
    MGK_CUDA(cudaGetLastError());
  }
  return MGK_OK;
}

extern "C" int mgk_ls2d_set_material_rep(mgk_ls2d_t p, int rep, const double* E, const double* nu,
                                         const double* epsp, mgk_stream_t stream) {
  MGK_REQUIRE(p && E && nu, "mgk_ls2d_set_material: null argument");
  MGK_REQUIRE(rep >= 0 && rep < p->nrep, "mgk_ls2d_set_material: replica %d out of range", rep);
  int st = ls2d_set_fields(p, rep, E, nu, epsp, 1, (cudaStream_t)stream);
  if (st == MGK_OK) p->has_material[rep] = 1;
  return st;
}

extern "C" int mgk_ls2d_set_material(mgk_ls2d_t p, const double* E, const double* nu, const double* epsp,
                                     mgk_stream_t stream) {
  return mgk_ls2d_set_material_rep(p, 0, E, nu, epsp, stream);
}

extern "C" int mgk_ls2d_set_lame_rep(mgk_ls2d_t p, int rep, const double* lam, const double* mu,
                                     const double* epsp, mgk_stream_t stream) {
  MGK_REQUIRE(p && lam && mu, "mgk_ls2d_set_lame: null argument");
  MGK_REQUIRE(rep >= 0 && rep < p->nrep, "mgk_ls2d_set_lame: replica %d out of range", rep);
  int st = ls2d_set_fields(p, rep, lam, mu, epsp, 2, (cudaStream_t)stream);
  if (st == MGK_OK) p->has_material[rep] = 1;
  return st;
}

// switches every replica of the plan to law (a, b, ps); cached loop graphs
// hold the previous law's row kernel and are dropped
static int ls2d_set_law(mgk_ls2d_t p, int law, double a, double b, int ps, const double* lp = nullptr) {
  for (auto& R : p->reps) {
    R.law = law; R.law_a = a; R.law_b = b; R.law_ps = ps;
    for (int q = 0; q < 11; ++q) R.lp[q] = lp ? lp[q] : 0.0;
  }
  p->law_a = a; p->law_b = b; p->law_ps = ps;
  if (law != p->law) {
    for (auto& e : p->gcache) {
      cudaGraphExecDestroy(e.x);
      cudaGraphDestroy(e.g);
    }
    p->gcache.clear();
    p->graph = nullptr;
    p->exec = nullptr;
    p->sel_rows = p->sel_cols = p->nsel = 0;  // the next solve builds its graph again
    if (p->graph_mode == 1) p->graph_mode = -1;
    p->law = law;
  }
  return MGK_OK;
}

extern "C" int mgk_ls2d_set_secant(mgk_ls2d_t p, double d, double k) {
  MGK_REQUIRE(p, "mgk_ls2d_set_secant: null plan");
  MGK_REQUIRE(d >= 0.0 && d <= 1.0 && k >= 0.0 && isfinite(k), "mgk_ls2d_set_secant: need 0 <= d <= 1, k >= 0");
  MGK_REQUIRE(d == 0.0 || p->prec == MGK_FP64, "mgk_ls2d_set_secant: the secant law runs in FP64 plans only");
  return ls2d_set_law(p, d != 0.0 ? 1 : 0, d, k, 0);
}

extern "C" int mgk_ls2d_set_rose(mgk_ls2d_t p, double eta, double floor_fraction, int plane_stress) {
  MGK_REQUIRE(p, "mgk_ls2d_set_rose: null plan");
  MGK_REQUIRE(eta >= 0.0 && isfinite(eta) && floor_fraction >= 0.0 && floor_fraction <= 1.0,
              "mgk_ls2d_set_rose: need eta >= 0, 0 <= floor_fraction <= 1");
  MGK_REQUIRE(p->prec == MGK_FP64, "mgk_ls2d_set_rose: the Rose law runs in FP64 plans only");
  return ls2d_set_law(p, 2, eta, floor_fraction, plane_stress ? 1 : 0);
}

extern "C" int mgk_ls2d_set_landau(mgk_ls2d_t p, const double* v, int capping, double e_cap, double tangent_ratio,
                                   double smooth_power, int plane_stress) {
  MGK_REQUIRE(p && v, "mgk_ls2d_set_landau: null argument");
  MGK_REQUIRE(p->prec == MGK_FP64, "mgk_ls2d_set_landau: the Landau law runs in FP64 plans only");
  MGK_REQUIRE(capping >= 0 && capping <= 2, "mgk_ls2d_set_landau: capping must be 0, 1 or 2");
  MGK_REQUIRE(!capping || (e_cap > 0.0 && isfinite(e_cap) && isfinite(tangent_ratio) &&
                           (capping != 2 || (smooth_power > 0.0 && isfinite(smooth_power)))),
              "mgk_ls2d_set_landau: need e_cap > 0 (and smooth_power > 0 for smooth capping)");
  double lp[11];
  for (int q = 0; q < 7; ++q) {
    MGK_REQUIRE(isfinite(v[q]), "mgk_ls2d_set_landau: non-finite coefficient");
    lp[q] = v[q];
  }
  lp[7] = capping; lp[8] = e_cap; lp[9] = tangent_ratio; lp[10] = smooth_power;
  return ls2d_set_law(p, 3, 0.0, 0.0, plane_stress ? 1 : 0, lp);
}

extern "C" int mgk_ls2d_set_e33_out(mgk_ls2d_t p, int rep, double* e33) {
  MGK_REQUIRE(p && rep >= 0 && rep < p->nrep, "mgk_ls2d_set_e33_out: bad argument");
  p->reps[rep].out_e33 = e33;
  return MGK_OK;
}

extern "C" int mgk_ls2d_set_anderson(mgk_ls2d_t p, int m) {
  MGK_REQUIRE(p, "mgk_ls2d_set_anderson: null plan");
  MGK_REQUIRE(m >= 0 && m <= kAaMax, "mgk_ls2d_set_anderson: depth must be 0..%d", kAaMax);
  MGK_REQUIRE(m == 0 || p->prec == MGK_FP64, "mgk_ls2d_set_anderson: Anderson mixing runs in FP64 plans only");
  if (m == p->aa_m) return MGK_OK;
  int rc = staging_wait(p);
  if (rc) return rc;
  // loop graphs hold the ring's address: rebuild them
  for (auto& e : p->gcache) {
    cudaGraphExecDestroy(e.x);
    cudaGraphDestroy(e.g);
  }
  p->gcache.clear();
  p->graph = nullptr;
  p->exec = nullptr;
  p->sel_rows = p->sel_cols = p->nsel = 0;
  if (p->graph_mode == 1) p->graph_mode = -1;
  if (m > 0) {
    const size_t need = (size_t)(3 + 2 * m) * 3 * (size_t)p->maxN;
    if (need > p->aa_doubles) {
      MGK_CUDA(cudaDeviceSynchronize());  // the old ring may be in use by queued work
      if (p->aa_buf) cudaFree(p->aa_buf);
      p->aa_buf = nullptr;
      p->aa_doubles = 0;
      if (cudaMalloc((void**)&p->aa_buf, need * sizeof(double)) != cudaSuccess) {
        cudaGetLastError();
        p->aa_buf = nullptr;
        p->aa_m = 0;
        set_error("mgk_ls2d_set_anderson: cudaMalloc of %zu bytes failed", need * sizeof(double));
        return MGK_OOM;
      }
      p->aa_doubles = need;
    }
    if (!p->d_aa) {
      int dev = 0, sms = 148;
      if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
      p->aa_nb = std::max(1, std::min(8 * sms, ceil_div(3 * p->maxN, kAaThreads)));
      if (cudaMalloc((void**)&p->d_aa, sizeof(Ls2dAA)) != cudaSuccess ||
          cudaMalloc((void**)&p->aa_part, sizeof(double) * 2 * kAaMax * p->aa_nb) != cudaSuccess) {
        cudaGetLastError();
        set_error("mgk_ls2d_set_anderson: cudaMalloc failed");
        p->aa_m = 0;
        return MGK_OOM;
      }
    }
  }
  p->aa_m = m;
  return MGK_OK;
}

extern "C" int mgk_ls2d_set_eigenstrain_rep(mgk_ls2d_t p, int rep, const double* epsp, mgk_stream_t stream) {
  MGK_REQUIRE(p && rep >= 0 && rep < p->nrep && p->has_material[rep],
              "mgk_ls2d_set_eigenstrain: replica has no material");
  return ls2d_set_fields(p, rep, nullptr, nullptr, epsp, 0, (cudaStream_t)stream);
}

extern "C" int mgk_ls2d_set_eigenstrain(mgk_ls2d_t p, const double* epsp, mgk_stream_t stream) {
  return mgk_ls2d_set_eigenstrain_rep(p, 0, epsp, stream);
}

// ------------------------------------------------------------- the loop ---

struct LoopArgs {
  const Ls2dRep* reps;
  Ls2dState* st;
  const int* row_map;
  const int* row_local;
  const int* col_map;
  const int* col_local;
  double* part;
  unsigned int* repctr;
  Ls2dCtl* ctl;
  int rows, cols;
  size_t row_smem, col_smem;
  int tma;            // use the persistent bulk-prefetch row kernel
  int row_grid;       // its grid (resident CTAs), <= rows
  int stage_bytes;
  size_t tma_smem;
  int fast;           // warp-line iteration kernels
  int law = 0;        // constitutive law of the warp-line row kernel (1: secant, 2: Rose, 3: Landau)
  // Anderson mixing (FP64 loop of a one-replica selection; aa_m = 0: none)
  int aa_m = 0;
  int aa_nb = 0;
  double* aa_buf = nullptr;
  Ls2dAA* aa = nullptr;
  double* aa_part = nullptr;
  const int* sel = nullptr;
};

template <typename TS, bool IN_SPEC, bool FINAL>
static void launch_row(const LoopArgs& a, cudaStream_t s) {
  if (a.fast) {
    void* fn = row_fast_fn<TS, IN_SPEC, FINAL>(a.fast, a.law);
    cudaGraphConditionalHandle h = 0;
    int zero = 0;
    void* args[] = {(void*)&a.reps, (void*)&a.st, (void*)&a.row_map, (void*)&a.row_local, (void*)&a.part,
                    (void*)&a.repctr, (void*)&a.ctl, &h, &zero, &zero};
    cudaLaunchKernel(fn, dim3(a.rows), dim3(row_threads(a.fast)), args, a.row_smem, s);
  } else {
    ls2d_row_kernel<TS, TS, IN_SPEC, FINAL><<<a.rows, kThreads, a.row_smem, s>>>(
        a.reps, a.st, a.row_map, a.row_local, a.part, a.repctr, a.ctl, 0, 0, 0);
  }
}

template <typename TS>
static void launch_col(const LoopArgs& a, cudaStream_t s) {
  if (a.fast) {
    void* fn = col_fast_fn<TS>(a.fast);
    void* args[] = {(void*)&a.reps, (void*)&a.st, (void*)&a.col_map, (void*)&a.col_local};
    cudaLaunchKernel(fn, dim3(a.cols), dim3(col_threads(a.fast)), args, a.col_smem, s);
  } else {
    ls2d_col_kernel<TS, TS><<<a.cols, kThreads, a.col_smem, s>>>(a.reps, a.st, a.col_map, a.col_local);
  }
}

// the history kernel of depth m (1..kAaMax)
static void* aa_update_fn(int m) {
  switch (m) {
    case 1: return (void*)ls2d_aa_update_kernel<1>;
    case 2: return (void*)ls2d_aa_update_kernel<2>;
    case 3: return (void*)ls2d_aa_update_kernel<3>;
    case 4: return (void*)ls2d_aa_update_kernel<4>;
    case 5: return (void*)ls2d_aa_update_kernel<5>;
    case 6: return (void*)ls2d_aa_update_kernel<6>;
    case 7: return (void*)ls2d_aa_update_kernel<7>;
    default: return (void*)ls2d_aa_update_kernel<8>;
  }
}

template <typename TS, bool FINAL>
static int launch_body(const LoopArgs& a, cudaStream_t s) {
  launch_col<TS>(a, s);
  MGK_CUDA(cudaGetLastError());
  if (a.tma)
    ls2d_row_tma_kernel<TS, TS, FINAL><<<a.row_grid, kThreads, a.tma_smem, s>>>(
        a.reps, a.st, a.row_map, a.row_local, a.part, a.repctr, a.ctl, 0, 0, 0, a.rows, a.stage_bytes);
  else
    launch_row<TS, true, FINAL>(a, s);
  MGK_CUDA(cudaGetLastError());
  if (sizeof(TS) == 8 && a.aa_m > 0) {
    void* args[] = {(void*)&a.reps, (void*)&a.st, (void*)&a.sel, (void*)&a.aa_buf, (void*)&a.aa, (void*)&a.aa_m,
                    (void*)&a.aa_part};
    cudaLaunchKernel(aa_update_fn(a.aa_m), dim3(a.aa_nb), dim3(kAaThreads), args, 0, s);
    launch_row<TS, false, FINAL>(a, s);  // the mix and tau of the mixed iterate
    MGK_CUDA(cudaGetLastError());
  }
  return MGK_OK;
}

template <typename TS, bool FINAL>
static int add_while(cudaGraph_t g, cudaGraphNode_t* node, const cudaGraphNode_t* dep, int ndep, LoopArgs& a,
                     int* guard_cap) {
  cudaGraphConditionalHandle h;
  MGK_CUDA(cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault));
  // cudaGraphNodeParams has no default constructor in C++: zeroed storage
  alignas(cudaGraphNodeParams) unsigned char raw[sizeof(cudaGraphNodeParams)];
  memset(raw, 0, sizeof(raw));
  cudaGraphNodeParams& cp = *reinterpret_cast<cudaGraphNodeParams*>(raw);
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = h;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  MGK_CUDA(cudaGraphAddNode(node, g, dep, ndep, &cp));
  cudaGraph_t body = cp.conditional.phGraph_out[0];
  cudaKernelNodeParams k1;
  memset(&k1, 0, sizeof(k1));
  void* a1[] = {&a.reps, &a.st, &a.col_map, &a.col_local};
  k1.func = a.fast ? col_fast_fn<TS>(a.fast) : (void*)ls2d_col_kernel<TS, TS>;
  k1.gridDim = dim3(a.cols);
  k1.blockDim = dim3(a.fast ? col_threads(a.fast) : kThreads);
  k1.sharedMemBytes = (unsigned)a.col_smem;
  k1.kernelParams = a1;
  cudaGraphNode_t n1, n2;
  MGK_CUDA(cudaGraphAddKernelNode(&n1, body, nullptr, 0, &k1));
  int use_cond = 1;
  cudaKernelNodeParams k2;
  memset(&k2, 0, sizeof(k2));
  void* a2[] = {&a.reps, &a.st, &a.row_map, &a.row_local, &a.part, &a.repctr, &a.ctl, &h, &use_cond, guard_cap};
  void* a2t[] = {&a.reps, &a.st, &a.row_map, &a.row_local, &a.part, &a.repctr, &a.ctl, &h, &use_cond, guard_cap,
                 &a.rows, &a.stage_bytes};
  if (a.tma) {
    k2.func = (void*)ls2d_row_tma_kernel<TS, TS, FINAL>;
    k2.gridDim = dim3(a.row_grid);
    k2.sharedMemBytes = (unsigned)a.tma_smem;
    k2.kernelParams = a2t;
    k2.blockDim = dim3(kThreads);
  } else {
    k2.func = a.fast ? row_fast_fn<TS, true, FINAL>(a.fast, a.law) : (void*)ls2d_row_kernel<TS, TS, true, FINAL>;
    k2.gridDim = dim3(a.rows);
    k2.sharedMemBytes = (unsigned)a.row_smem;
    k2.kernelParams = a2;
    k2.blockDim = dim3(a.fast ? row_threads(a.fast) : kThreads);
  }
  MGK_CUDA(cudaGraphAddKernelNode(&n2, body, &n1, 1, &k2));
  if (sizeof(TS) == 8 && a.aa_m > 0) {
    // Anderson history and least squares, then the mix and tau of the mixed
    // iterate in the first row pass
    cudaGraphNode_t n3, n6;
    cudaKernelNodeParams k3, k6;
    memset(&k3, 0, sizeof(k3));
    memset(&k6, 0, sizeof(k6));
    void* a3[] = {&a.reps, &a.st, &a.sel, &a.aa_buf, &a.aa, &a.aa_m, &a.aa_part};
    k3.func = aa_update_fn(a.aa_m);
    k3.gridDim = dim3(a.aa_nb);
    k3.blockDim = dim3(kAaThreads);
    k3.kernelParams = a3;
    MGK_CUDA(cudaGraphAddKernelNode(&n3, body, &n2, 1, &k3));
    cudaGraphConditionalHandle h0 = 0;
    int zero = 0;
    void* a6[] = {&a.reps, &a.st, &a.row_map, &a.row_local, &a.part, &a.repctr, &a.ctl, &h0, &zero, &zero};
    k6.func = a.fast ? row_fast_fn<TS, false, FINAL>(a.fast, a.law) : (void*)ls2d_row_kernel<TS, TS, false, FINAL>;
    k6.gridDim = dim3(a.rows);
    k6.blockDim = dim3(a.fast ? row_threads(a.fast) : kThreads);
    k6.sharedMemBytes = (unsigned)a.row_smem;
    k6.kernelParams = a6;
    MGK_CUDA(cudaGraphAddKernelNode(&n6, body, &n3, 1, &k6));
  }
  return MGK_OK;
}

// Graph for the current selection: mixed plans run [phase-1 while, promote,
// phase-2 setup, first FP64 row kernel] before the final while node.  It is
// rebuilt when the selection's shape or the iteration cap changes.
static int build_graph(mgk_ls2d_t p, LoopArgs& a64, LoopArgs& a32, const int* d_sel, int nsel, int G,
                       int guard_cap) {
  cudaGraph_t g = nullptr;
  MGK_CUDA(cudaGraphCreate(&g, 0));
  int cap = guard_cap;
  int rc = MGK_OK;
  cudaGraphNode_t last;
  if (p->prec == MGK_MIXED) {
    cudaGraphNode_t w1, n_prom, n_ph2, n_row0;
    rc = add_while<float, false>(g, &w1, nullptr, 0, a32, &cap);
    if (rc == MGK_OK) {
      cudaKernelNodeParams k;
      memset(&k, 0, sizeof(k));
      void* ap[] = {&a64.reps, (void*)&d_sel};
      k.func = (void*)ls2d_promote_kernel;
      k.gridDim = dim3(G, nsel);
      k.blockDim = dim3(kThreads);
      k.kernelParams = ap;
      rc = cudaGraphAddKernelNode(&n_prom, g, &w1, 1, &k) == cudaSuccess ? MGK_OK : MGK_CUDA_ERROR;
    }
    if (rc == MGK_OK) {
      cudaKernelNodeParams k2;
      memset(&k2, 0, sizeof(k2));
      void* ap2[] = {&a64.st, (void*)&d_sel, &nsel, &a64.ctl};
      k2.func = (void*)ls2d_phase2_kernel;
      k2.gridDim = dim3(1);
      k2.blockDim = dim3(32);
      k2.kernelParams = ap2;
      rc = cudaGraphAddKernelNode(&n_ph2, g, &n_prom, 1, &k2) == cudaSuccess ? MGK_OK : MGK_CUDA_ERROR;
    }
    if (rc == MGK_OK) {
      cudaKernelNodeParams k3;
      memset(&k3, 0, sizeof(k3));
      cudaGraphConditionalHandle h0 = 0;
      int zero = 0;
      void* ap3[] = {&a64.reps, &a64.st, &a64.row_map, &a64.row_local, &a64.part, &a64.repctr, &a64.ctl,
                     &h0, &zero, &zero};
      k3.func = a64.fast ? row_fast_fn<double, false, true>(a64.fast, a64.law)
                         : (void*)ls2d_row_kernel<double, double, false, true>;
      k3.gridDim = dim3(a64.rows);
      k3.blockDim = dim3(a64.fast ? row_threads(a64.fast) : kThreads);
      k3.sharedMemBytes = (unsigned)a64.row_smem;
      k3.kernelParams = ap3;
      rc = cudaGraphAddKernelNode(&n_row0, g, &n_ph2, 1, &k3) == cudaSuccess ? MGK_OK : MGK_CUDA_ERROR;
    }
    if (rc == MGK_OK) rc = add_while<double, true>(g, &last, &n_row0, 1, a64, &cap);
  } else {
    rc = add_while<double, true>(g, &last, nullptr, 0, a64, &cap);
  }
  cudaGraphExec_t x = nullptr;
  if (rc == MGK_OK && cudaGraphInstantiate(&x, g, 0) != cudaSuccess) rc = MGK_CUDA_ERROR;
  if (rc != MGK_OK) {
    cudaGraphDestroy(g);
    cudaGetLastError();
    return rc;
  }
  constexpr size_t kMaxGraphs = 48;
  if (p->gcache.size() >= kMaxGraphs) {
    cudaGraphExecDestroy(p->gcache.front().x);
    cudaGraphDestroy(p->gcache.front().g);
    p->gcache.erase(p->gcache.begin());
  }
  p->gcache.push_back({a64.rows, a64.cols, nsel, guard_cap, a64.aa_m, g, x});
  p->graph = g;
  p->exec = x;
  return MGK_OK;
}

// Switches the plan's kernel family: 0 = CTA-wide passes, 256/512/1024 =
// warp-line kernels for sides up to that length (at least the plan's
// largest side).  Column tiles, shared-memory sizes and the cached loop
// graphs follow the family.
static int ls2d_set_variant(mgk_ls2d_t p, int v) {
  MGK_REQUIRE(v == 0 || (p->fast_nat && v >= p->fast_nat && (v == 256 || v == 512 || v == 1024)),
              "mgk_ls2d: kernel family %d cannot serve this plan", v);
  const size_t c64 = sizeof(double2);
  size_t rs = 0, cs = 0, rs32 = 0, cs32 = 0;
  int tot_cols = 0;
  for (int r = 0; r < p->nrep; ++r) {
    Ls2dRep& R = p->reps[r];
    R.tc = v ? fast_col_tiles(v) : p->tc_gen[r];
    R.col_items = (R.nyh + R.tc - 1) / R.tc;
    tot_cols += R.col_items;
    if (v) {
      rs = std::max(rs, (size_t)row_fast_smem(R.ny, 16, 8));
      cs = std::max(cs, (size_t)col_fast_smem(R.nx, 16, R.tc));
      rs32 = std::max(rs32, (size_t)row_fast_smem(R.ny, 8, 4));
      cs32 = std::max(cs32, (size_t)col_fast_smem(R.nx, 8, R.tc));
    } else {
      rs = std::max(rs, 2 * 3 * (size_t)R.ny * c64);
      cs = std::max(cs, 2 * 3 * (size_t)R.tc * R.nx * c64);
      rs32 = rs / 2;
      cs32 = cs / 2;
    }
  }
  int st = v ? ls2d_set_fast_attrs<double>(v, rs, cs) : ls2d_set_attrs<double, double>(rs, cs);
  if (st == MGK_OK && p->prec == MGK_MIXED)
    st = v ? ls2d_set_fast_attrs<float>(v, rs32, cs32) : ls2d_set_attrs<float, float>(rs32, cs32);
  if (st) return st;
  p->fast = v;
  p->total_col_items = tot_cols;
  p->row_smem = rs; p->col_smem = cs; p->row_smem32 = rs32; p->col_smem32 = cs32;
  for (auto& e : p->gcache) {
    cudaGraphExecDestroy(e.x);
    cudaGraphDestroy(e.g);
  }
  p->gcache.clear();
  p->graph = nullptr;
  p->exec = nullptr;
  p->graph_mode = -1;
  p->sel_rows = p->sel_cols = p->nsel = 0;
  return MGK_OK;
}

extern "C" int mgk_ls2d_profile_batch(mgk_ls2d_t p, int nsel, const int* sel, const double* eps_bar, int fp32,
                                      int reps, float* row_ms, float* col_ms, mgk_stream_t stream);

extern "C" int mgk_ls2d_set_family(mgk_ls2d_t p, int family) {
  MGK_REQUIRE(p, "mgk_ls2d_set_family: null plan");
  MGK_CUDA(cudaDeviceSynchronize());  // no loop graph of this plan in flight
  return ls2d_set_variant(p, family);
}

extern "C" int mgk_ls2d_autotune(mgk_ls2d_t p, int nsel, const int* sel, const double* eps_bar, int reps,
                                 int* chosen, float* best_ms, mgk_stream_t stream) {
  MGK_REQUIRE(p && eps_bar && nsel >= 1 && reps >= 1, "mgk_ls2d_autotune: bad argument");
  int cands[4];
  int nc = 0;
  if (p->fast_nat)
    for (int v : {256, 512, 1024})
      if (v >= p->fast_nat) cands[nc++] = v;
  cands[nc++] = 0;
  int best = p->fast;
  float best_t = 0.0f;
  for (int k = 0; k < nc; ++k) {
    int st = ls2d_set_variant(p, cands[k]);
    if (st) return st;
    float r64 = 0, c64 = 0, r32 = 0, c32 = 0;
    st = mgk_ls2d_profile_batch(p, nsel, sel, eps_bar, 0, reps, &r64, &c64, stream);
    if (st == MGK_OK && p->prec == MGK_MIXED) st = mgk_ls2d_profile_batch(p, nsel, sel, eps_bar, 1, reps, &r32, &c32, stream);
    if (st) return st;
    const float t = r64 + c64 + r32 + c32;
    if (k == 0 || t < best_t) { best_t = t; best = cands[k]; }
  }
  int st = ls2d_set_variant(p, best);
  if (st) return st;
  if (chosen) *chosen = best;
  if (best_ms) *best_ms = best_t;
  return MGK_OK;
}

// Copies the replicas' states to the host (one synchronisation of the
// stream) and fills infos for the selection.
static int ls2d_collect(mgk_ls2d_t p, int nsel, const int* selv, mgk_ls_info* infos, cudaStream_t s) {
  MGK_CUDA(cudaMemcpyAsync(p->h_state, p->d_st, sizeof(Ls2dState) * p->nrep, cudaMemcpyDeviceToHost, s));
  Ls2dCtl hc;
  MGK_CUDA(cudaMemcpyAsync(&hc, p->d_ctl, sizeof(Ls2dCtl), cudaMemcpyDeviceToHost, s));
  MGK_CUDA(cudaStreamSynchronize(s));
  if (hc.error) {
    set_error("mgk_ls2d_solve: a bulk copy wait gave up (device timeout)");
    return MGK_TIMEOUT;
  }
  int worst = MGK_OK;
  for (int q = 0; q < nsel; ++q) {
    const Ls2dState& S = p->h_state[selv[q]];
    infos[q].iterations = S.iter;
    infos[q].status = S.status;
    infos[q].final_diff = S.diff;
    for (int k = 0; k < 4; ++k) { infos[q].eps_mean[k] = S.out_eps_mean[k]; infos[q].sig_mean[k] = S.out_sig_mean[k]; }
    if (S.status == MGK_NONFINITE) worst = MGK_NONFINITE;
  }
  if (worst == MGK_NONFINITE) {
    set_error("mgk_ls2d_solve: non-finite residual");
    return MGK_NONFINITE;
  }
  return MGK_OK;
}

extern "C" int mgk_ls2d_collect(mgk_ls2d_t p, int nsel, const int* sel, mgk_ls_info* infos, mgk_stream_t stream) {
  MGK_REQUIRE(p && sel && infos && nsel >= 1 && nsel <= p->nrep, "mgk_ls2d_collect: bad argument");
  for (int q = 0; q < nsel; ++q)
    MGK_REQUIRE(sel[q] >= 0 && sel[q] < p->nrep, "mgk_ls2d_collect: replica %d out of range", sel[q]);
  return ls2d_collect(p, nsel, sel, infos, (cudaStream_t)stream);
}

extern "C" int mgk_ls2d_solve_batch(mgk_ls2d_t p, int nsel, const int* sel, const double* eps_bar,
                                    const double* const* eps_init, double* const* eps_out, double* const* sig_out,
                                    int max_iter, double tol, mgk_ls_info* infos, mgk_stream_t stream) {
  MGK_REQUIRE(p && eps_bar && nsel >= 1 && nsel <= p->nrep, "mgk_ls2d_solve_batch: bad argument");
  MGK_REQUIRE(max_iter >= 0 && max_iter <= 1000000, "mgk_ls2d_solve: max_iter out of range");
  MGK_REQUIRE(p->aa_m == 0 || nsel == 1, "mgk_ls2d_solve_batch: Anderson mixing solves one replica per call");
  MGK_REQUIRE(p->aa_m == 0 || p->law != 0, "mgk_ls2d_solve_batch: Anderson mixing runs with a nonlinear law");
  cudaStream_t s = (cudaStream_t)stream;
  std::vector<int> selv(nsel);
  std::vector<char> seen(p->nrep, 0);
  for (int q = 0; q < nsel; ++q) {
    const int r = sel ? sel[q] : q;
    MGK_REQUIRE(r >= 0 && r < p->nrep && !seen[r], "mgk_ls2d_solve_batch: bad or repeated replica index");
    MGK_REQUIRE(p->has_material[r], "mgk_ls2d_solve: replica %d has no material (call set_material)", r);
    // the Rose law reads the [0,1] strain entry; the symmetric storage carries it
    // when macro strain and eigenstrain are symmetric (the eigenstrain is the
    // caller's to keep symmetric)
    MGK_REQUIRE(p->law < 2 || eps_bar[4 * q + 1] == eps_bar[4 * q + 2],
                "mgk_ls2d_solve: the Rose and Landau laws need a symmetric macro strain");
    seen[r] = 1;
    selv[q] = r;
  }
  int rc = staging_wait(p);
  if (rc) return rc;
  // per-call fields and compact work maps
  int rows = 0, cols = 0;
  for (int q = 0; q < nsel; ++q) { rows += p->reps[selv[q]].row_items; cols += p->reps[selv[q]].col_items; }
  const bool changed = rows != p->sel_rows || cols != p->sel_cols || nsel != p->nsel || p->aa_m != p->graph_aa;
  int* row_map = p->h_maps;
  int* row_local = row_map + rows;
  int* col_map = row_local + rows;
  int* col_local = col_map + cols;
  int* selp = col_local + cols;
  int ri = 0, ci = 0;
  for (int q = 0; q < nsel; ++q) {
    const int r = selv[q];
    Ls2dRep& H = p->h_reps[r];
    H = p->reps[r];
    H.init = eps_init ? eps_init[q] : nullptr;
    H.out_eps = eps_out ? eps_out[q] : nullptr;
    H.out_sig = sig_out ? sig_out[q] : nullptr;
    for (int k = 0; k < 4; ++k) H.eb[k] = eps_bar[4 * q + k];
    H.tol = tol;
    H.max_iter = max_iter;
    H.aa = p->aa_m > 0 ? p->d_aa : nullptr;
    H.aa_x = p->aa_m > 0 ? p->aa_buf : nullptr;
    H.aa_dG = p->aa_m > 0 ? p->aa_buf + (size_t)(3 + p->aa_m) * 3 * (size_t)H.N : nullptr;
    H.row_first = ri;
    H.col_first = ci;
    for (int i = 0; i < H.row_items; ++i) { row_map[ri] = r; row_local[ri] = i; ++ri; }
    for (int i = 0; i < H.col_items; ++i) { col_map[ci] = r; col_local[ci] = i; ++ci; }
    selp[q] = r;
  }
  const int n_active = max_iter > 0 ? nsel : 0;
  p->h_ctl->n_active = (unsigned int)n_active;
  p->h_ctl->decided = 0;
  p->h_ctl->still = 0;
  p->h_ctl->bodies = 0;
  p->h_ctl->any = n_active > 0;
  p->h_ctl->error = 0;
  const size_t nm = 2 * (size_t)rows + 2 * (size_t)cols + nsel;
  MGK_CUDA(cudaMemcpyAsync(p->d_maps, p->h_maps, sizeof(int) * nm, cudaMemcpyHostToDevice, s));
  MGK_CUDA(cudaMemcpyAsync(p->d_reps, p->h_reps, sizeof(Ls2dRep) * p->nrep, cudaMemcpyHostToDevice, s));
  MGK_CUDA(cudaMemcpyAsync(p->d_ctl, p->h_ctl, sizeof(Ls2dCtl), cudaMemcpyHostToDevice, s));
  MGK_CUDA(cudaEventRecord(p->staged, s));
  p->staged_pending = true;
  p->sel_rows = rows;
  p->sel_cols = cols;
  p->nsel = nsel;

  const int* d_row_map = p->d_maps;
  const int* d_row_local = d_row_map + rows;
  const int* d_col_map = d_row_local + rows;
  const int* d_col_local = d_col_map + cols;
  const int* d_sel = d_col_local + cols;
  const int G = grid_blocks(p->maxN);
  bool any_init = false;
  for (int q = 0; q < nsel && eps_init; ++q) any_init |= eps_init[q] != nullptr;
  if (any_init) {
    ls2d_means_kernel<<<dim3(G, nsel), kThreads, 0, s>>>(p->d_reps, d_sel, p->d_part);
    MGK_CUDA(cudaGetLastError());
    ls2d_finalize_kernel<<<nsel, kThreads, 0, s>>>(p->d_reps, p->d_st, d_sel, p->d_part, G, 4,
                                                   (int)offsetof(Ls2dState, means), 1);
    MGK_CUDA(cudaGetLastError());
  }
  ls2d_begin_kernel<<<dim3(G, nsel), kThreads, 0, s>>>(p->d_reps, p->d_st, d_sel, p->d_part);
  MGK_CUDA(cudaGetLastError());
  if (any_init) {
    ls2d_finalize_kernel<<<nsel, kThreads, 0, s>>>(p->d_reps, p->d_st, d_sel, p->d_part, G, 2,
                                                   (int)offsetof(Ls2dState, extra_d0), 2);
    MGK_CUDA(cudaGetLastError());
  }
  if (n_active > 0) {
    const bool mixed = p->prec == MGK_MIXED;
    LoopArgs a64{p->d_reps, p->d_st, d_row_map, d_row_local, d_col_map, d_col_local, p->d_part, p->d_repctr,
                 p->d_ctl, rows, cols, p->row_smem, p->col_smem, p->tma, 0, p->stage64, p->tma_smem64, p->fast};
    a64.row_grid = std::max(1, std::min(rows, p->occ64 * p->num_sms));
    a64.law = p->law;
    LoopArgs a32 = a64;
    a32.law = 0;
    if (p->aa_m > 0) {
      a64.aa_m = p->aa_m;
      a64.aa_nb = p->aa_nb;
      a64.aa_buf = p->aa_buf;
      a64.aa = p->d_aa;
      a64.aa_part = p->aa_part;
      a64.sel = d_sel;
      ls2d_aa_init_kernel<<<p->aa_nb, kThreads, 0, s>>>(p->d_reps, d_sel, p->aa_buf, p->d_aa);
      MGK_CUDA(cudaGetLastError());
    }
    a32.row_smem = p->row_smem32;
    a32.col_smem = p->col_smem32;
    a32.stage_bytes = p->stage32;
    a32.tma_smem = p->tma_smem32;
    a32.row_grid = std::max(1, std::min(rows, p->occ32 * p->num_sms));
    if (mixed) launch_row<float, false, false>(a32, s);
    else launch_row<double, false, true>(a64, s);
    MGK_CUDA(cudaGetLastError());
    const int guard_cap = (max_iter + 2 > 1000 ? max_iter + 2 : 1000);
    if (p->graph_mode == 1 && (changed || guard_cap > p->graph_cap)) {
      bool hit = false;
      for (auto& e : p->gcache)
        if (e.rows == rows && e.cols == cols && e.nsel == nsel && e.cap >= guard_cap && e.aa == p->aa_m) {
          p->graph = e.g;
          p->exec = e.x;
          p->graph_cap = e.cap;
          p->graph_aa = e.aa;
          hit = true;
          break;
        }
      if (!hit) p->graph_mode = -1;
    }
    if (p->graph_mode < 0) {
      const char* env = getenv("MGK_NO_GRAPH_WHILE");
      if (env && env[0] == '1') p->graph_mode = 0;
      else {
        p->graph_mode = build_graph(p, a64, a32, d_sel, nsel, G, guard_cap) == MGK_OK ? 1 : 0;
        p->graph_cap = guard_cap;
        p->graph_aa = p->aa_m;
      }
    }
    if (p->graph_mode == 1) {
      MGK_CUDA(cudaGraphLaunch(p->exec, s));
    } else {
      // host-driven loop: poll the device flag after each iteration
      for (int phase = mixed ? 1 : 2; phase <= 2; ++phase) {
        if (phase == 2 && mixed) {
          ls2d_promote_kernel<<<dim3(G, nsel), kThreads, 0, s>>>(p->d_reps, d_sel);
          ls2d_phase2_kernel<<<1, 32, 0, s>>>(p->d_st, d_sel, nsel, p->d_ctl);
          launch_row<double, false, true>(a64, s);
          MGK_CUDA(cudaGetLastError());
        }
        for (int it = 0; it < max_iter; ++it) {
          rc = (phase == 1) ? launch_body<float, false>(a32, s) : launch_body<double, true>(a64, s);
          if (rc) return rc;
          Ls2dCtl hc;
          MGK_CUDA(cudaMemcpyAsync(&hc, p->d_ctl, sizeof(Ls2dCtl), cudaMemcpyDeviceToHost, s));
          MGK_CUDA(cudaStreamSynchronize(s));
          if (!hc.any) break;
        }
      }
    }
  }
  if (p->law == 1) ls2d_output_kernel<1><<<dim3(G, nsel), kThreads, 0, s>>>(p->d_reps, p->d_st, d_sel, p->d_part);
  else if (p->law == 2) ls2d_output_kernel<2><<<dim3(G, nsel), kThreads, 0, s>>>(p->d_reps, p->d_st, d_sel, p->d_part);
  else if (p->law == 3) ls2d_output_kernel<3><<<dim3(G, nsel), kThreads, 0, s>>>(p->d_reps, p->d_st, d_sel, p->d_part);
  else ls2d_output_kernel<<<dim3(G, nsel), kThreads, 0, s>>>(p->d_reps, p->d_st, d_sel, p->d_part);
  MGK_CUDA(cudaGetLastError());
  ls2d_finalize_kernel<<<nsel, kThreads, 0, s>>>(p->d_reps, p->d_st, d_sel, p->d_part, G, 8,
                                                 (int)offsetof(Ls2dState, out_eps_mean), 0);
  MGK_CUDA(cudaGetLastError());
  if (infos) return ls2d_collect(p, nsel, selv.data(), infos, s);
  return MGK_OK;
}

extern "C" int mgk_ls2d_solve(mgk_ls2d_t p, const double* eps_bar, const double* eps_init, double* eps_out,
                              double* sig_out, int max_iter, double tol, mgk_ls_info* info, mgk_stream_t stream) {
  MGK_REQUIRE(p && eps_bar, "mgk_ls2d_solve: null argument");
  int r0 = 0;
  return mgk_ls2d_solve_batch(p, 1, &r0, eps_bar, &eps_init, &eps_out, &sig_out, max_iter, tol, info, stream);
}

// ----------------------------------------------------------- profiling ---

template <typename TS>
static int profile_t(mgk_ls2d_t p, float* row_ms, float* col_ms, int reps, cudaStream_t s) {
  const int rows = p->sel_rows, cols = p->sel_cols;
  const int* d_row_map = p->d_maps;
  const int* d_row_local = d_row_map + rows;
  const int* d_col_map = d_row_local + rows;
  const int* d_col_local = d_col_map + cols;
  const size_t rs = sizeof(TS) == 8 ? p->row_smem : p->row_smem32;
  const size_t cs = sizeof(TS) == 8 ? p->col_smem : p->col_smem32;
  LoopArgs a{p->d_reps, p->d_st, d_row_map, d_row_local, d_col_map, d_col_local, p->d_part, p->d_repctr,
             p->d_ctl, rows, cols, rs, cs, 0, 0, 0, 0, p->fast};
  a.law = sizeof(TS) == 8 ? p->law : 0;
  launch_row<TS, false, true>(a, s);
  MGK_CUDA(cudaGetLastError());
  cudaEvent_t ev[3];
  for (int i = 0; i < 3; ++i) MGK_CUDA(cudaEventCreate(&ev[i]));
  float tr = 0, tc = 0;
  int rc = MGK_OK;
  for (int r = 0; r < reps; ++r) {
    cudaEventRecord(ev[0], s);
    launch_col<TS>(a, s);
    cudaEventRecord(ev[1], s);
    if (p->tma) {
      const bool f64 = sizeof(TS) == 8;
      const int grid = std::max(1, std::min(rows, (f64 ? p->occ64 : p->occ32) * p->num_sms));
      ls2d_row_tma_kernel<TS, TS, true><<<grid, kThreads, f64 ? p->tma_smem64 : p->tma_smem32, s>>>(
          p->d_reps, p->d_st, d_row_map, d_row_local, p->d_part, p->d_repctr, p->d_ctl, 0, 0, 0, rows,
          f64 ? p->stage64 : p->stage32);
    } else {
      launch_row<TS, true, true>(a, s);
    }
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

extern "C" int mgk_ls2d_profile_batch(mgk_ls2d_t p, int nsel, const int* sel, const double* eps_bar, int fp32,
                                      int reps, float* row_ms, float* col_ms, mgk_stream_t stream) {
  MGK_REQUIRE(p && eps_bar && row_ms && col_ms && reps > 0, "mgk_ls2d_profile: bad argument");
  MGK_REQUIRE(!fp32 || p->prec == MGK_MIXED, "mgk_ls2d_profile: FP32 kernels need a mixed-precision plan");
  cudaStream_t s = (cudaStream_t)stream;
  // set up the selection with a zero-iteration solve, then time iterations
  // with tolerance 0 and an unreachable cap so every replica stays active
  std::vector<const double*> init(nsel, nullptr);
  std::vector<double*> outs(nsel, nullptr);
  int rc = mgk_ls2d_solve_batch(p, nsel, sel, eps_bar, init.data(), outs.data(), outs.data(), 0, 0.0, nullptr,
                                stream);
  if (rc) return rc;
  rc = staging_wait(p);
  if (rc) return rc;
  for (int q = 0; q < nsel; ++q) {
    Ls2dRep& H = p->h_reps[sel ? sel[q] : q];
    H.max_iter = 1 << 30;
    H.tol = 0.0;
  }
  MGK_CUDA(cudaMemcpyAsync(p->d_reps, p->h_reps, sizeof(Ls2dRep) * p->nrep, cudaMemcpyHostToDevice, s));
  for (int q = 0; q < nsel; ++q) {
    const int r = sel ? sel[q] : q;
    MGK_CUDA(cudaMemsetAsync(reinterpret_cast<char*>(&p->d_st[r]) + offsetof(Ls2dState, done), 0, sizeof(int), s));
  }
  p->h_ctl->n_active = nsel;
  p->h_ctl->decided = 0;
  p->h_ctl->still = 0;
  p->h_ctl->bodies = 0;
  MGK_CUDA(cudaMemcpyAsync(p->d_ctl, p->h_ctl, sizeof(Ls2dCtl), cudaMemcpyHostToDevice, s));
  MGK_CUDA(cudaStreamSynchronize(s));
  return fp32 ? profile_t<float>(p, row_ms, col_ms, reps, s) : profile_t<double>(p, row_ms, col_ms, reps, s);
}

extern "C" int mgk_ls2d_profile(mgk_ls2d_t p, const double* eps_bar, int reps, float* row_ms, float* col_ms,
                                mgk_stream_t stream) {
  int r0 = 0;
  return mgk_ls2d_profile_batch(p, 1, &r0, eps_bar, 0, reps, row_ms, col_ms, stream);
}

// ------------------------------------------------- one-voxel eigenstrain ---

namespace mgk {
// Copy voxel (x, y) = d_xy[0..1] of the caller's eigenstrain field (after a
// flip) into the plan's planes; a negative x means no event happened.
__global__ void ls2d_sync_voxel_kernel(const Ls2dRep* reps, int rep, const double* __restrict__ epsp,
                                       const long long* __restrict__ d_xy) {
  const long long x = d_xy[0], y = d_xy[1];
  const Ls2dRep& R = reps[rep];
  if (x < 0 || y < 0 || x >= R.nx || y >= R.ny) return;
  const long long N = R.N, i = x * R.ny + y;
  const double4 p = reinterpret_cast<const double4*>(epsp)[i];
  const double psym = (p.y == p.z) ? p.y : 0.5 * (p.y + p.z);
  R.ep[i] = p.x;
  R.ep[N + i] = p.w;
  R.ep[2 * N + i] = psym;
  if (R.ep32) { R.ep32[i] = (float)p.x; R.ep32[N + i] = (float)p.w; R.ep32[2 * N + i] = (float)psym; }
  if (R.epa) { R.epa[i] = p.y; R.epa[N + i] = p.z; }
}
}  // namespace mgk

extern "C" int mgk_ls2d_sync_voxel(mgk_ls2d_t p, int rep, const double* eps_plastic, const int64_t* d_xy,
                                   mgk_stream_t stream) {
  MGK_REQUIRE(p && eps_plastic && d_xy && rep >= 0 && rep < p->nrep && p->has_material[rep],
              "mgk_ls2d_sync_voxel: bad argument");
  MGK_REQUIRE(p->reps[rep].epa != nullptr, "mgk_ls2d_sync_voxel: set the material with an eigenstrain field first");
  ls2d_sync_voxel_kernel<<<1, 1, 0, (cudaStream_t)stream>>>(p->d_reps, rep, eps_plastic, (const long long*)d_xy);
  MGK_CUDA(cudaGetLastError());
  return MGK_OK;
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
constexpr size_t kNaMisc = 1024;                    // plan record, state, control, work maps
constexpr size_t kNaDoubles = kNaPlanes + kNaSpec + kNaTw + kNaPart + kNaMisc;
// byte offsets inside the misc region
constexpr size_t kNaRep = 0, kNaState = 1024, kNaCtl = 2048, kNaCtr = 2112, kNaMaps = 2176;
constexpr int kNaMapInts = 128 + 128 + 256 + 256 + 1;
static_assert(kNaMaps + 4 * kNaMapInts <= kNaMisc * sizeof(double), "no-alloc misc region");
}  // namespace

// Device-side storage.  In host code this name is only a stand-in for the
// device address, which cudaGetSymbolAddress resolves per device.
static __device__ __align__(256) double g_ls2d_noalloc_scratch[kNaDoubles];

namespace mgk {

// Writes the plan record and the work maps, clears the state, the control
// block and the arrival counter, and fills the twiddle tables (sincospi):
// everything a call must start from.
__global__ void ls2d_noalloc_setup_kernel(Ls2dRep rep, Ls2dRep* dst, Ls2dState* st, Ls2dCtl* ctl,
                                          unsigned int* repctr, int* maps, int rows, int cols, int n_active,
                                          double2* twx, int nx, double2* twy, int ny) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int stride = gridDim.x * blockDim.x;
  int* row_map = maps;
  int* row_local = row_map + rows;
  int* col_map = row_local + rows;
  int* col_local = col_map + cols;
  int* sel = col_local + cols;
  for (int i = t; i < rows; i += stride) { row_map[i] = 0; row_local[i] = i; }
  for (int i = t; i < cols; i += stride) { col_map[i] = 0; col_local[i] = i; }
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
    sel[0] = 0;
    *repctr = 0;
    Ls2dState z;
    memset(&z, 0, sizeof(z));
    *st = z;
    ctl->n_active = (unsigned int)n_active;
    ctl->decided = 0;
    ctl->still = 0;
    ctl->bodies = 0;
    ctl->any = n_active > 0;
  }
}

}  // namespace mgk

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
  MGK_REQUIRE(nx >= 2 && ny >= 1 && nx <= MGK_NOALLOC_MAX_SIDE && ny <= MGK_NOALLOC_MAX_SIDE,
              "mgk_ls2d_solve_noalloc: grid %dx%d exceeds the maximum of %dx%d for the allocation-free entry "
              "point (use mgk_ls2d_create/mgk_ls2d_solve)", nx, ny, MGK_NOALLOC_MAX_SIDE, MGK_NOALLOC_MAX_SIDE);
  FftLen fx, fy;
  MGK_REQUIRE(fft_schedule(nx, &fx) && fft_schedule(ny, &fy) && nx % 2 == 0,
              "mgk_ls2d_solve_noalloc: grid %dx%d unsupported (each side 2^a 3^b, nx even)", nx, ny);
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
  const int tc = pick_tc(nx, sizeof(double2), 64 * 1024);
  const int rows = nx / 2, cols = (nyh + tc - 1) / tc;
  const size_t row_smem = 2 * 3 * (size_t)ny * sizeof(double2);
  const size_t col_smem = 2 * 3 * (size_t)tc * nx * sizeof(double2);
  st = ls2d_set_attrs<double, double>(row_smem, col_smem);
  if (st != MGK_OK) return st;

  // carve the scratch array (offsets in doubles, each region 256-byte aligned)
  double* planes = base;
  double2* spec = reinterpret_cast<double2*>(base + kNaPlanes);
  double2* twx = reinterpret_cast<double2*>(base + kNaPlanes + kNaSpec);
  double2* twy = twx + MGK_NOALLOC_MAX_SIDE;
  double* part = base + kNaPlanes + kNaSpec + kNaTw;
  char* misc = reinterpret_cast<char*>(base + kNaPlanes + kNaSpec + kNaTw + kNaPart);
  Ls2dRep* d_rep = reinterpret_cast<Ls2dRep*>(misc + kNaRep);
  Ls2dState* d_st = reinterpret_cast<Ls2dState*>(misc + kNaState);
  Ls2dCtl* d_ctl = reinterpret_cast<Ls2dCtl*>(misc + kNaCtl);
  unsigned int* d_ctr = reinterpret_cast<unsigned int*>(misc + kNaCtr);
  int* d_maps = reinterpret_cast<int*>(misc + kNaMaps);
  static_assert(sizeof(Ls2dRep) <= 1024 && sizeof(Ls2dState) <= 1024 && sizeof(Ls2dCtl) <= 64,
                "no-alloc record sizes");
  const int* d_row_map = d_maps;
  const int* d_row_local = d_row_map + rows;
  const int* d_col_map = d_row_local + rows;
  const int* d_col_local = d_col_map + cols;
  const int* d_sel = d_col_local + cols;

  fx.tw = twx;
  fy.tw = twy;
  Ls2dRep R;
  memset(&R, 0, sizeof(R));
  R.nx = nx; R.ny = ny; R.nyh = nyh; R.ld = nyh; R.tc = tc;
  R.row_items = rows; R.col_items = cols;
  R.N = N; R.fx64 = fx; R.fy64 = fy; R.fx32 = fx; R.fy32 = fy;
  R.mu = planes; R.lam = planes + N; R.eps = planes + 2 * N; R.ep = planes + 5 * N;
  R.epa = eps_plastic ? planes + 8 * N : nullptr;
  R.spec = spec;
  R.init = eps_init; R.out_eps = eps_out; R.out_sig = sig_out;
  for (int k = 0; k < 4; ++k) R.eb[k] = eps_bar[k];
  R.tol = tol; R.max_iter = max_iter; R.row_first = 0; R.col_first = 0;

  ls2d_noalloc_setup_kernel<<<4, 256, 0, s>>>(R, d_rep, d_st, d_ctl, d_ctr, d_maps, rows, cols,
                                              max_iter > 0 ? 1 : 0, twx, nx, twy, ny);
  MGK_CUDA(cudaGetLastError());
  const int G = grid_blocks(N);
  ls2d_material_kernel<<<G, kThreads, 0, s>>>(d_rep, 0, E, nu, eps_plastic, plane_mode, 1, part);
  MGK_CUDA(cudaGetLastError());
  ls2d_medium_kernel<<<1, kThreads, 0, s>>>(d_rep, d_st, 0, part, G, plane_mode, 0, 0.0);
  MGK_CUDA(cudaGetLastError());
  if (eps_init) {
    ls2d_means_kernel<<<dim3(G, 1), kThreads, 0, s>>>(d_rep, d_sel, part);
    ls2d_finalize_kernel<<<1, kThreads, 0, s>>>(d_rep, d_st, d_sel, part, G, 4, (int)offsetof(Ls2dState, means), 1);
    MGK_CUDA(cudaGetLastError());
  }
  ls2d_begin_kernel<<<dim3(G, 1), kThreads, 0, s>>>(d_rep, d_st, d_sel, part);
  MGK_CUDA(cudaGetLastError());
  if (eps_init) {
    ls2d_finalize_kernel<<<1, kThreads, 0, s>>>(d_rep, d_st, d_sel, part, G, 2, (int)offsetof(Ls2dState, extra_d0),
                                                1);
    MGK_CUDA(cudaGetLastError());
  }
  if (max_iter > 0) {
    ls2d_row_kernel<double, double, false, true><<<rows, kThreads, row_smem, s>>>(
        d_rep, d_st, d_row_map, d_row_local, part, d_ctr, d_ctl, 0, 0, 0);
    MGK_CUDA(cudaGetLastError());
    // host-driven loop in chunks of 4 iterations; finished replicas skip
    // their work on the device, and the host polls the activity flag
    LoopArgs a{d_rep, d_st, d_row_map, d_row_local, d_col_map, d_col_local, part, d_ctr, d_ctl, rows, cols,
               row_smem, col_smem};
    int it = 0;
    while (it < max_iter) {
      const int chunk = max_iter - it < 4 ? max_iter - it : 4;
      for (int c = 0; c < chunk; ++c) {
        st = launch_body<double, true>(a, s);
        if (st != MGK_OK) return st;
      }
      it += chunk;
      Ls2dCtl hc;
      MGK_CUDA(cudaMemcpyAsync(&hc, d_ctl, sizeof(Ls2dCtl), cudaMemcpyDeviceToHost, s));
      MGK_CUDA(cudaStreamSynchronize(s));
      if (!hc.any) break;
    }
  }
  ls2d_output_kernel<<<dim3(G, 1), kThreads, 0, s>>>(d_rep, d_st, d_sel, part);
  MGK_CUDA(cudaGetLastError());
  ls2d_finalize_kernel<<<1, kThreads, 0, s>>>(d_rep, d_st, d_sel, part, G, 8, (int)offsetof(Ls2dState, out_eps_mean),
                                              0);
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

extern "C" int64_t mgk_aa_work_bytes(int64_t n) {
  (void)n;
  return (int64_t)sizeof(double) * kAaBlocks * 2 * kAaMax;
}

extern "C" int mgk_aa_update(int64_t n, const double* x, const double* g, double* hist, int m, int slot,
                             int have_prev, int ncols, double* dots, void* work, mgk_stream_t stream) {
  MGK_REQUIRE(n > 0 && x && g && hist && work && dots, "mgk_aa_update: bad argument");
  MGK_REQUIRE(m >= 1 && m <= kAaMax && ncols >= 0 && ncols <= m && slot >= 0 && slot < m &&
                  (!have_prev || slot < ncols),
              "mgk_aa_update: need 1 <= m <= %d, 0 <= ncols <= m, slot < m (and < ncols with a previous pair)",
              kAaMax);
  cudaStream_t s = (cudaStream_t)stream;
  const int nb = (int)std::min<long long>(kAaBlocks, (n + 255) / 256);
  double* part = reinterpret_cast<double*>(work);
  aa_update_kernel<<<nb, 256, 0, s>>>(n, x, g, hist, m, slot, have_prev, ncols, part);
  MGK_CUDA(cudaGetLastError());
  if (ncols > 0) {
    aa_sum_kernel<<<1, 256, 0, s>>>(part, nb, ncols, dots);
    MGK_CUDA(cudaGetLastError());
  }
  return MGK_OK;
}

extern "C" int mgk_aa_mix(int64_t n, const double* g, const double* hist, int m, int ncols, const double* gamma,
                          double* x, mgk_stream_t stream) {
  MGK_REQUIRE(n > 0 && g && hist && x && (ncols == 0 || gamma), "mgk_aa_mix: bad argument");
  MGK_REQUIRE(m >= 1 && m <= kAaMax && ncols >= 0 && ncols <= m, "mgk_aa_mix: need 1 <= m <= %d, ncols <= m",
              kAaMax);
  AaCoef c;
  for (int j = 0; j < kAaMax; ++j) {
    c.v[j] = j < ncols ? gamma[j] : 0.0;
    MGK_REQUIRE(isfinite(c.v[j]), "mgk_aa_mix: non-finite coefficient");
  }
  const int nb = (int)std::min<long long>(4 * kAaBlocks, (n + 255) / 256);
  aa_mix_kernel<<<nb, 256, 0, (cudaStream_t)stream>>>(n, g, hist, m, ncols, c, x);
  MGK_CUDA(cudaGetLastError());
  return MGK_OK;
}
