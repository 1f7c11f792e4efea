// STDE reductions on the device.
//
// The Taylor sweep writes c2 for every (point, direction) unit; these kernels
// turn them into per-point EstimatorResults with the reference's Welford
// accumulator (src/stde/types.rs:44-113): non-finite samples are skipped, the
// mean is NaN when nothing contributed, the variance m2/(n-1) is clamped at 0
// and the standard error is sqrt(var/n).  Samples are visited in direction
// order, as the reference's host loop does (src/gpu/stde_gpu.rs:84-97).
//
// Accumulator precision: `Acc` = the sample type for the drop-in calls (so an
// f32 laplacian_gpu reproduces the reference's f32 Welford exactly), and double
// for the batched extension (FP64 final reduction of FP32 samples).
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/echidna_b200.h"
#include "launch.h"
#include "rng.cuh"

namespace ech {

template <class Acc>
struct Welford {
  Acc mean = Acc(0), m2 = Acc(0);
  uint64_t count = 0;
  __device__ void update(Acc s) {
    if (!isfinite(s)) return;
    count += 1;
    const Acc k1 = (Acc)count;
    const Acc delta = s - mean;
    mean = mean + delta / k1;
    const Acc delta2 = s - mean;
    m2 = m2 + delta * delta2;
  }
  __device__ void finalize(Acc* est, Acc* var, Acc* se) const {
    if (count == 0) {
      *est = __longlong_as_double(0x7ff8000000000000ll);
      *var = Acc(0);
      *se = Acc(0);
      return;
    }
    const Acc nf = (Acc)count;
    if (count > 1) {
      const Acc v = fmax(m2 / (nf - Acc(1)), Acc(0));
      *est = mean;
      *var = v;
      *se = sqrt(v / nf);
    } else {
      *est = mean;
      *var = Acc(0);
      *se = Acc(0);
    }
  }
};

// One thread per point: samples scale*c_k of units [p*S, (p+1)*S) (scale 2,
// k = 2 for the Laplacian; k!, k for k-th order diagonals), optionally minus a
// control term cv[s] plus `trace` (laplacian_with_control).
// With `wmul`, each sample is also multiplied by its unit's weight (importance
// sampling: 1 / p of the sampled coordinate).
template <class T, class Acc>
__global__ void stde_reduce_kernel(const T* c0, const T* ck, T scale, uint64_t npoints, uint32_t S, const T* cv,
                                   T trace, int control, const T* wmul, ech_estimator_result* out) {
  const uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npoints) return;
  Welford<Acc> acc;
  for (uint32_t s = 0; s < S; ++s) {
    T vhv = scale * ck[p * S + s];
    if (wmul) vhv = vhv * wmul[p * S + s];
    if (control) acc.update((Acc)(vhv - cv[s]));
    else acc.update((Acc)vhv);
  }
  Acc est, var, se;
  acc.finalize(&est, &var, &se);
  ech_estimator_result r;
  // every direction of a point shares the primal; report the first's c0
  // (src/gpu/stde_gpu.rs:88 reads values[0])
  r.value = (double)c0[p * S];
  r.estimate = control ? (double)((T)trace + (T)est) : (double)est;
  r.sample_variance = (double)var;
  r.standard_error = (double)se;
  r.num_samples = acc.count;
  out[p] = r;
}

// Neumaier's compensated summation (Neumaier, 1974): the running sum s plus
// the accumulated rounding errors c.
template <class T>
struct Neumaier {
  T s = T(0), c = T(0);
  __device__ __forceinline__ void add(T x) {
    const T t = s + x;
    if (fabs(s) >= fabs(x)) c = c + ((s - t) + x);
    else c = c + ((x - t) + s);
    s = t;
  }
  __device__ __forceinline__ T value() const { return s + c; }
};

// The batch extension's compensated FP32 reduction, one thread per point: the
// mean of the finite samples from a compensated sum, then the corrected
// two-pass variance (Chan, Golub and LeVeque, 1983) from compensated sums of
// the deviations and of their squares.  Count, NaN mean at count 0, the clamp
// at 0 and the standard error are as in the Welford reduction.
template <class T>
__global__ void stde_reduce_comp_kernel(const T* c0, const T* ck, T scale, uint64_t npoints, uint32_t S,
                                        const T* wmul, ech_estimator_result* out) {
  const uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npoints) return;
  Neumaier<T> sum;
  uint64_t count = 0;
  for (uint32_t s = 0; s < S; ++s) {
    T x = scale * ck[p * S + s];
    if (wmul) x = x * wmul[p * S + s];
    if (!isfinite(x)) continue;
    sum.add(x);
    count += 1;
  }
  ech_estimator_result r;
  r.value = (double)c0[p * S];
  r.num_samples = count;
  if (count == 0) {
    r.estimate = __longlong_as_double(0x7ff8000000000000ll);
    r.sample_variance = 0.0;
    r.standard_error = 0.0;
    out[p] = r;
    return;
  }
  const T nf = (T)count;
  const T mean = sum.value() / nf;
  T var = T(0);
  if (count > 1) {
    Neumaier<T> dev, sq;
    for (uint32_t s = 0; s < S; ++s) {
      T x = scale * ck[p * S + s];
      if (wmul) x = x * wmul[p * S + s];
      if (!isfinite(x)) continue;
      const T d = x - mean;
      dev.add(d);
      sq.add(d * d);
    }
    const T dv = dev.value();
    var = fmax((sq.value() - dv * dv / nf) / (nf - T(1)), T(0));
  }
  r.estimate = (double)mean;
  r.sample_variance = (double)var;
  r.standard_error = (double)sqrt(var / nf);
  out[p] = r;
}

cudaError_t launch_stde_reduce_comp(const void* c0, const void* ck, double scale, uint64_t npoints, uint32_t S,
                                    const void* wmul, void* results, cudaStream_t st) {
  const int threads = 128;
  const unsigned blocks = (unsigned)((npoints + threads - 1) / threads);
  if (blocks == 0) return cudaSuccess;
  stde_reduce_comp_kernel<float><<<blocks, threads, 0, st>>>((const float*)c0, (const float*)ck, (float)scale, npoints,
                                                             S, (const float*)wmul, (ech_estimator_result*)results);
  return cudaGetLastError();
}

// stde_sparse (src/stde/sparse.rs:37-78), per point: for each sampled entry e
// in order, raw = c_{k_e} * prefactor_e and sample = sign_e * Z * raw, Welford in
// the sample type; the value is c0 of the point's last sample.  Coefficients
// are coefficient-major, coeffs[k * units + u] (one scalar output).
template <class T>
__global__ void stde_sparse_reduce_kernel(const T* coeffs, uint64_t units, const uint32_t* ent, const uint32_t* kout,
                                          const T* pref, const T* sign, T z, uint64_t npoints, uint32_t S,
                                          ech_estimator_result* out) {
  const uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npoints) return;
  Welford<T> acc;
  T value = T(0);
  for (uint32_t s = 0; s < S; ++s) {
    const uint64_t u = p * S + s;
    const uint32_t e = ent[u];
    value = coeffs[u];
    const T raw = coeffs[(uint64_t)kout[e] * units + u] * pref[e];
    const T sample = sign[e] * z * raw;
    acc.update(sample);
  }
  T est, var, se;
  acc.finalize(&est, &var, &se);
  ech_estimator_result r;
  r.value = (double)value;
  r.estimate = (double)est;
  r.sample_variance = (double)var;
  r.standard_error = (double)se;
  r.num_samples = acc.count;
  out[p] = r;
}

cudaError_t launch_stde_sparse_reduce(bool f64, const void* coeffs, uint64_t units, const uint32_t* ent,
                                      const uint32_t* kout, const void* pref, const void* sign, double z,
                                      uint64_t npoints, uint32_t S, void* results, cudaStream_t st) {
  const int threads = 128;
  const unsigned blocks = (unsigned)((npoints + threads - 1) / threads);
  if (blocks == 0) return cudaSuccess;
  if (f64)
    stde_sparse_reduce_kernel<double><<<blocks, threads, 0, st>>>((const double*)coeffs, units, ent, kout,
                                                                  (const double*)pref, (const double*)sign, z,
                                                                  npoints, S, (ech_estimator_result*)results);
  else
    stde_sparse_reduce_kernel<float><<<blocks, threads, 0, st>>>((const float*)coeffs, units, ent, kout,
                                                                 (const float*)pref, (const float*)sign, (float)z,
                                                                 npoints, S, (ech_estimator_result*)results);
  return cudaGetLastError();
}

// v^T diag(H) v per direction, summed in index order in T (src/gpu/stde_gpu.rs:178-184).
template <class T>
__global__ void control_term_kernel(const T* dirs, const T* diag, uint32_t S, uint32_t n, T* cv) {
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= S) return;
  T acc = T(0);
  for (uint32_t j = 0; j < n; ++j) {
    const T vj = dirs[(uint64_t)s * n + j];
    acc = acc + diag[j] * vj * vj;
  }
  cv[s] = acc;
}

cudaError_t launch_stde_reduce_t(bool f64, bool acc64, const void* c0, const void* c2, double scale, uint64_t npoints,
                                 uint32_t S, const void* cv, double trace, int control, const void* wmul,
                                 void* results, cudaStream_t st) {
  const int threads = 128;
  const unsigned blocks = (unsigned)((npoints + threads - 1) / threads);
  if (blocks == 0) return cudaSuccess;
  if (f64) {
    stde_reduce_kernel<double, double><<<blocks, threads, 0, st>>>((const double*)c0, (const double*)c2, scale, npoints, S,
                                                                   (const double*)cv, trace, control, (const double*)wmul,
                                                                   (ech_estimator_result*)results);
  } else if (acc64) {
    stde_reduce_kernel<float, double><<<blocks, threads, 0, st>>>((const float*)c0, (const float*)c2, (float)scale,
                                                                  npoints, S,
                                                                  (const float*)cv, (float)trace, control, (const float*)wmul,
                                                                  (ech_estimator_result*)results);
  } else {
    stde_reduce_kernel<float, float><<<blocks, threads, 0, st>>>((const float*)c0, (const float*)c2, (float)scale,
                                                                 npoints, S,
                                                                 (const float*)cv, (float)trace, control, (const float*)wmul,
                                                                 (ech_estimator_result*)results);
  }
  return cudaGetLastError();
}

cudaError_t launch_control_term(bool f64, const void* dirs, const void* diag, uint32_t S, uint32_t n, void* cv,
                                cudaStream_t st) {
  const int threads = 128;
  const unsigned blocks = (S + threads - 1) / threads;
  if (blocks == 0) return cudaSuccess;
  if (f64)
    control_term_kernel<double><<<blocks, threads, 0, st>>>((const double*)dirs, (const double*)diag, S, n, (double*)cv);
  else
    control_term_kernel<float><<<blocks, threads, 0, st>>>((const float*)dirs, (const float*)diag, S, n, (float*)cv);
  return cudaGetLastError();
}

// Coordinate sampling for sparse STDE: one block per point draws S coordinates
// from the row of `probs` (inverse CDF of the row's prefix sums) or uniformly
// (probs == nullptr), with Philox uniforms keyed by (seed, point, sample), and
// records each sample's importance weight total / p_j (n for uniform draws).
template <class T>
__global__ void sample_coords_kernel(const float* probs, uint32_t n, uint64_t npoints, uint32_t S, uint64_t seed,
                                     uint32_t* idx, T* wmul) {
  extern __shared__ double cdf[];
  const uint64_t pt = blockIdx.x;
  if (pt >= npoints) return;
  const float* row = probs ? probs + pt * n : nullptr;
  if (row && threadIdx.x == 0) {
    double acc = 0.0;
    for (uint32_t j = 0; j < n; ++j) {
      acc += (double)row[j];
      cdf[j] = acc;
    }
  }
  __syncthreads();
  const double total = row ? cdf[n - 1] : 1.0;
  for (uint32_t s = threadIdx.x; s < S; s += blockDim.x) {
    const double u = (double)philox_uniform(seed, pt, s, 0);
    uint32_t j;
    T w;
    if (row) {
      const double target = u * total;
      uint32_t lo = 0, hi = n - 1;  // first j with cdf[j] > target
      while (lo < hi) {
        const uint32_t mid = (lo + hi) / 2;
        if (cdf[mid] > target) hi = mid;
        else lo = mid + 1;
      }
      j = lo;
      const double pj = fmax((double)row[j], 1e-30) / total;
      w = (T)(1.0 / pj);
    } else {
      j = min((uint32_t)(u * (double)n), n - 1);
      w = (T)n;
    }
    idx[pt * S + s] = j;
    wmul[pt * S + s] = w;
  }
}

template <class T>
__global__ void scale_kernel(T* y, T a, size_t n) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) y[i] = a * y[i];
}

cudaError_t launch_sample_coords(bool f64, const float* probs, uint32_t n, uint64_t npoints, uint32_t S,
                                 uint64_t seed, uint32_t* idx, void* wmul, cudaStream_t st) {
  if (npoints == 0) return cudaSuccess;
  const size_t smem = probs ? (size_t)n * sizeof(double) : 0;
  if (smem > 48 * 1024) {
    cudaError_t e = f64 ? cudaFuncSetAttribute(sample_coords_kernel<double>,
                                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)
                        : cudaFuncSetAttribute(sample_coords_kernel<float>,
                                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  if (f64)
    sample_coords_kernel<double><<<(unsigned)npoints, 128, smem, st>>>(probs, n, npoints, S, seed, idx, (double*)wmul);
  else
    sample_coords_kernel<float><<<(unsigned)npoints, 128, smem, st>>>(probs, n, npoints, S, seed, idx, (float*)wmul);
  return cudaGetLastError();
}

cudaError_t launch_scale(bool f64, void* y, double a, size_t n, cudaStream_t st) {
  const unsigned blocks = (unsigned)((n + 255) / 256);
  if (blocks == 0) return cudaSuccess;
  if (f64) scale_kernel<double><<<blocks, 256, 0, st>>>((double*)y, a, n);
  else scale_kernel<float><<<blocks, 256, 0, st>>>((float*)y, (float)a, n);
  return cudaGetLastError();
}

}  // namespace ech
