// Library-wide runtime pieces: error text, status names, FFT schedules and
// the per-device twiddle-table cache.
#include <stdarg.h>

#include <map>
#include <tuple>
#include <mutex>
#include <vector>
#include <cmath>

#include "common.cuh"
#include "fft.cuh"

namespace mgk {

static thread_local char g_err[2048] = "";

void set_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}

cudaError_t raise_smem(const void* fn, size_t bytes) {
  static std::mutex m;
  static std::map<std::pair<int, const void*>, size_t> set;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> g(m);
  size_t& cur = set[{dev, fn}];
  if (bytes <= cur) return cudaSuccess;
  e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (e == cudaSuccess) cur = bytes;
  return e;
}

bool fft_schedule(int n, FftLen* f) {
  if (n < 1 || n > 4096) return false;
  int m = n, a = 0, b = 0;
  while (m % 3 == 0) { m /= 3; ++b; }
  while (m % 2 == 0) { m /= 2; ++a; }
  if (m != 1) return false;
  int np = 0;
  for (int i = 0; i < b; ++i) f->radix[np++] = 3;
  int p8 = a / 3, rem = a % 3;
  if (rem == 1 && p8 >= 1) { p8 -= 1; rem = 4; }  // 2^(3k+1) = 8^(k-1) * 4 * 4
  for (int i = 0; i < p8; ++i) f->radix[np++] = 8;
  if (rem == 4) { f->radix[np++] = 4; f->radix[np++] = 4; }
  else if (rem == 2) f->radix[np++] = 4;
  else if (rem == 1) f->radix[np++] = 2;
  if (np > 8) return false;
  f->n = n;
  f->npass = np;
  f->tw = nullptr;
  return true;
}

// Twiddle tables W_n^m = exp(-2 pi i m / n), one per (device, n, precision);
// they live until process exit (a few tens of KB in total).
const void* twiddles(int n, int prec) {
  static std::mutex mu;
  static std::map<std::tuple<int, int, int>, void*> cache;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
  std::lock_guard<std::mutex> lock(mu);
  auto key = std::make_tuple(dev, n, prec);
  auto it = cache.find(key);
  if (it != cache.end()) return it->second;
  void* d = nullptr;
  const size_t bytes = (size_t)n * (prec == MGK_FP64 ? sizeof(double2) : sizeof(float2));
  if (cudaMalloc(&d, bytes) != cudaSuccess) return nullptr;
  if (prec == MGK_FP64) {
    std::vector<double2> h(n);
    for (int m = 0; m < n; ++m) {
      long double ang = -2.0L * 3.14159265358979323846264338327950288L * (long double)m / (long double)n;
      h[m].x = (double)cosl(ang);
      h[m].y = (double)sinl(ang);
    }
    if (cudaMemcpy(d, h.data(), bytes, cudaMemcpyHostToDevice) != cudaSuccess) return nullptr;
  } else {
    std::vector<float2> h(n);
    for (int m = 0; m < n; ++m) {
      long double ang = -2.0L * 3.14159265358979323846264338327950288L * (long double)m / (long double)n;
      h[m].x = (float)cosl(ang);
      h[m].y = (float)sinl(ang);
    }
    if (cudaMemcpy(d, h.data(), bytes, cudaMemcpyHostToDevice) != cudaSuccess) return nullptr;
  }
  cache[key] = d;
  return d;
}

}  // namespace mgk

extern "C" {

int mgk_version(void) { return 100; }

const char* mgk_status_string(int s) {
  switch (s) {
    case MGK_OK: return "ok";
    case MGK_NOT_CONVERGED: return "not converged";
    case MGK_NONFINITE: return "non-finite value";
    case MGK_BAD_ARG: return "bad argument";
    case MGK_OOM: return "out of device memory";
    case MGK_TIMEOUT: return "timeout";
    case MGK_CUDA_ERROR: return "CUDA error";
    default: return "unknown status";
  }
}

const char* mgk_last_error(void) { return mgk::g_err; }

int mgk_fft_supported(int n) {
  mgk::FftLen f;
  return mgk::fft_schedule(n, &f) ? 1 : 0;
}

}  // extern "C"
