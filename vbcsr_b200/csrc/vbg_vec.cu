// Multivector / vector operations on device buffers: scale, axpby, bdot,
// pointwise products and the counter-based random fill.
//
// Reference behaviour replaced:
//   DistMultiVector::scale/axpy/axpby/pointwise_mult/bdot
//     vbcsr/core/dist_multivector.hpp:179-314
//   DistVector::dot  vbcsr/core/dist_vector.hpp:113
//   set_random       vbcsr/core/dist_multivector.hpp:335-373 with the entry
//                    generator of vbcsr/core/random_vectors.hpp:52-160
#include <algorithm>
#include <cmath>

#include "vbg_internal.cuh"

namespace vbg {

static int vgrid(int64_t n, int threads = 256) {
  int64_t g = (n + threads - 1) / threads;
  g = std::min<int64_t>(g, (int64_t)sm_count() * 16);
  return (int)std::max<int64_t>(g, 1);
}

template <typename T>
__device__ __forceinline__ T cmul(T a, double re, double im);
template <>
__device__ __forceinline__ double cmul<double>(double a, double re, double) { return a * re; }
template <>
__device__ __forceinline__ cplx cmul<cplx>(cplx a, double re, double im) {
  return {a.re * re - a.im * im, a.re * im + a.im * re};
}

// Element (row, col < k) of an n_rows x ld buffer; pad lanes are left alone.
template <typename T>
__global__ void mv_scale_kernel(int64_t n_rows, int k, int ld, double re, double im, T* X) {
  const int64_t total = n_rows * k;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = i / k;
    const int c = (int)(i - r * k);
    X[r * ld + c] = cmul(X[r * ld + c], re, im);
  }
}

template <typename T>
__global__ void mv_axpby_kernel(int64_t n_rows, int k, int ld, double are, double aim, const T* X, double bre,
                                double bim, T* Y) {
  const int64_t total = n_rows * k;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = i / k;
    const int c = (int)(i - r * k);
    const int64_t j = r * ld + c;
    const T ax = cmul(X[j], are, aim);
    const T by = cmul(Y[j], bre, bim);
    if constexpr (sizeof(T) == sizeof(cplx)) {
      Y[j] = ax + by;
    } else {
      Y[j] = ax + by;
    }
  }
}

template <typename T>
__global__ void mv_pointwise_kernel(int64_t n_rows, int k, int ld, const T* Yv, int y_is_vector, T* X) {
  const int64_t total = n_rows * k;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = i / k;
    const int c = (int)(i - r * k);
    const T y = y_is_vector ? Yv[r] : Yv[r * ld + c];
    const T x = X[r * ld + c];
    if constexpr (sizeof(T) == sizeof(cplx)) {
      const cplx a = *reinterpret_cast<const cplx*>(&x), b = *reinterpret_cast<const cplx*>(&y);
      cplx z{a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
      X[r * ld + c] = *reinterpret_cast<T*>(&z);
    } else {
      X[r * ld + c] = x * y;
    }
  }
}

// Per-column dots: each CTA reduces a row range into partial[cta][k] (k <= 128
// per pass), a second kernel sums the CTA partials in order.
template <typename T>
__global__ void bdot_partial_kernel(int64_t n_rows, int k, int ld, int c0, int kc, const T* X, const T* Y, T* part) {
  extern __shared__ unsigned char smem_raw[];
  T* acc = reinterpret_cast<T*>(smem_raw);  // [blockDim.x]
  // threads laid out as (row lane) x (column): column = tid % kc
  const int tid = threadIdx.x;
  const int rows_per_pass = blockDim.x / kc;
  const int c = tid % kc;
  const int rl = tid / kc;
  T sum;
  if constexpr (sizeof(T) == sizeof(cplx)) sum = T{0.0, 0.0}; else sum = T(0);
  if (rl < rows_per_pass) {
    for (int64_t r = blockIdx.x * (int64_t)rows_per_pass + rl; r < n_rows; r += (int64_t)gridDim.x * rows_per_pass) {
      const T a = X[r * ld + c0 + c];
      const T b = Y[r * ld + c0 + c];
      if constexpr (sizeof(T) == sizeof(cplx)) {
        sum.re = fma(a.re, b.re, fma(a.im, b.im, sum.re));
        sum.im = fma(a.re, b.im, fma(-a.im, b.re, sum.im));
      } else {
        sum = fma(a, b, sum);
      }
    }
  }
  acc[tid] = sum;
  __syncthreads();
  if (tid < kc) {
    T s = acc[tid];
    for (int j = 1; j < rows_per_pass; ++j) s = s + acc[tid + j * kc];
    part[(int64_t)blockIdx.x * kc + tid] = s;
  }
}

template <typename T>
__global__ void bdot_final_kernel(int nparts, int kc, int c0, const T* part, T* out) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= kc) return;
  T s = part[c];
  for (int p = 1; p < nparts; ++p) s = s + part[(int64_t)p * kc + c];
  out[c0 + c] = s;
}

// ---------------------------------------------------------------- random
// splitmix64 counter hash (Steele, Lea & Flood, OOPSLA 2014), mixed one key
// field at a time: seed, global block id, row inside the block, column.
__device__ __forceinline__ uint64_t splitmix64(uint64_t x) {
  x += 0x9e3779b97f4a7c15ULL;
  x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ULL;
  x = (x ^ (x >> 27)) * 0x94d049bb133111ebULL;
  return x ^ (x >> 31);
}
__device__ __forceinline__ uint64_t entry_hash(uint64_t seed, uint64_t block, uint64_t row, uint64_t col) {
  uint64_t h = splitmix64(seed + 0x9e3779b97f4a7c15ULL);
  h = splitmix64(h ^ (block * 0xbf58476d1ce4e5b9ULL));
  h = splitmix64(h ^ (row * 0x94d049bb133111ebULL));
  return splitmix64(h ^ (col * 0xd6e8feb86659fd93ULL));
}

// One warp per block row; lanes over (row-in-block, column) pairs.
template <typename T>
__global__ void set_random_kernel(int n, const int* __restrict__ bsz, const int64_t* __restrict__ scal_off, int k,
                                  int ld, uint64_t seed, double scale, T* X) {
  const int lane = threadIdx.x & 31;
  const int warps = blockDim.x >> 5;
  for (int b = blockIdx.x * warps + (threadIdx.x >> 5); b < n; b += gridDim.x * warps) {
    const int r = bsz[b];
    const int64_t row0 = scal_off[b];
    for (int p = lane; p < r * k; p += 32) {
      const int t = p / k, c = p - (p / k) * k;
      const uint64_t h = entry_hash(seed, (uint64_t)b, (uint64_t)t, (uint64_t)c);
      if constexpr (sizeof(T) == sizeof(cplx)) {
        // random phase exp(i theta), theta = 2 pi u, u from the top 53 bits
        const double u = (double)(h >> 11) * (1.0 / 9007199254740992.0);
        const double theta = 2.0 * 3.14159265358979323846 * u;
        double sv, cv;
        sincos(theta, &sv, &cv);
        cplx z{cv * scale, sv * scale};
        X[(row0 + t) * ld + c] = *reinterpret_cast<T*>(&z);
      } else {
        // Rademacher: the sign is the hash's top bit
        const double v = (h >> 63) ? 1.0 : -1.0;
        X[(row0 + t) * ld + c] = v * scale;
      }
    }
  }
}

template <typename T>
static int bdot_t(int64_t n_rows, int k, int ld, const T* X, const T* Y, T* out, cudaStream_t s) {
  constexpr int threads = 256;
  const int nparts = std::max(1, std::min<int>(sm_count() * 2, (int)((n_rows + 63) / 64)));
  DevBuf part;
  int rc = part.ensure((size_t)nparts * std::min(k, 128) * sizeof(T));
  if (rc) return rc;
  for (int c0 = 0; c0 < k; c0 += 128) {
    const int kc = std::min(128, k - c0);
    bdot_partial_kernel<T><<<nparts, threads, threads * sizeof(T), s>>>(n_rows, k, ld, c0, kc, X, Y, part.as<T>());
    bdot_final_kernel<T><<<(kc + 127) / 128, 128, 0, s>>>(nparts, kc, c0, part.as<T>(), out);
  }
  VBG_CUDA(cudaGetLastError());
  // part is released when this returns; keep the stream ordered against the free.
  VBG_CUDA(cudaStreamSynchronize(s));
  return 0;
}

}  // namespace vbg

using namespace vbg;

extern "C" {

int vbg_mv_scale(int dtype, int64_t n_rows, int k, int ld, double re, double im, void* X, void* stream) {
  VBG_CHECK(X || n_rows == 0, VBG_E_ARG, "null buffer");
  VBG_CHECK(k >= 1 && ld >= k, VBG_E_ARG, "invalid k / ld");
  if (n_rows == 0) return 0;
  cudaStream_t s = as_stream(stream);
  if (dtype == VBG_C128)
    mv_scale_kernel<cplx><<<vgrid(n_rows * k), 256, 0, s>>>(n_rows, k, ld, re, im, static_cast<cplx*>(X));
  else
    mv_scale_kernel<double><<<vgrid(n_rows * k), 256, 0, s>>>(n_rows, k, ld, re, im, static_cast<double*>(X));
  VBG_CUDA(cudaGetLastError());
  return 0;
}

int vbg_mv_axpby(int dtype, int64_t n_rows, int k, int ld, double are, double aim, const void* X, double bre,
                 double bim, void* Y, void* stream) {
  VBG_CHECK((X && Y) || n_rows == 0, VBG_E_ARG, "null buffer");
  VBG_CHECK(k >= 1 && ld >= k, VBG_E_ARG, "invalid k / ld");
  if (n_rows == 0) return 0;
  cudaStream_t s = as_stream(stream);
  if (dtype == VBG_C128)
    mv_axpby_kernel<cplx><<<vgrid(n_rows * k), 256, 0, s>>>(n_rows, k, ld, are, aim, static_cast<const cplx*>(X),
                                                              bre, bim, static_cast<cplx*>(Y));
  else
    mv_axpby_kernel<double><<<vgrid(n_rows * k), 256, 0, s>>>(n_rows, k, ld, are, aim,
                                                                static_cast<const double*>(X), bre, bim,
                                                                static_cast<double*>(Y));
  VBG_CUDA(cudaGetLastError());
  return 0;
}

int vbg_mv_pointwise(int dtype, int64_t n_rows, int k, int ld, const void* Yv, int y_is_vector, void* X,
                     void* stream) {
  VBG_CHECK((X && Yv) || n_rows == 0, VBG_E_ARG, "null buffer");
  VBG_CHECK(k >= 1 && ld >= k, VBG_E_ARG, "invalid k / ld");
  if (n_rows == 0) return 0;
  cudaStream_t s = as_stream(stream);
  if (dtype == VBG_C128)
    mv_pointwise_kernel<cplx><<<vgrid(n_rows * k), 256, 0, s>>>(n_rows, k, ld, static_cast<const cplx*>(Yv),
                                                                  y_is_vector, static_cast<cplx*>(X));
  else
    mv_pointwise_kernel<double><<<vgrid(n_rows * k), 256, 0, s>>>(n_rows, k, ld, static_cast<const double*>(Yv),
                                                                    y_is_vector, static_cast<double*>(X));
  VBG_CUDA(cudaGetLastError());
  return 0;
}

int vbg_mv_bdot(int dtype, int64_t n_rows, int k, int ld, const void* X, const void* Y, void* out, void* stream) {
  VBG_CHECK(X && Y && out, VBG_E_ARG, "null buffer");
  VBG_CHECK(k >= 1 && ld >= k, VBG_E_ARG, "invalid k / ld");
  cudaStream_t s = as_stream(stream);
  if (n_rows == 0) {
    VBG_CUDA(cudaMemsetAsync(out, 0, (size_t)k * elem_size(dtype), s));
    return 0;
  }
  if (dtype == VBG_C128)
    return bdot_t<cplx>(n_rows, k, ld, static_cast<const cplx*>(X), static_cast<const cplx*>(Y),
                        static_cast<cplx*>(out), s);
  return bdot_t<double>(n_rows, k, ld, static_cast<const double*>(X), static_cast<const double*>(Y),
                        static_cast<double*>(out), s);
}

int vbg_mv_set_random(const vbg_matrix* m, int k, int ld, uint64_t seed, int normalize, void* X, void* stream) {
  VBG_CHECK(m && X, VBG_E_ARG, "null argument");
  VBG_CHECK(k >= 1 && ld >= k, VBG_E_ARG, "invalid k / ld");
  if (m->n == 0) return 0;
  cudaStream_t s = as_stream(stream);
  // Unit-modulus draws have |v|^2 = N exactly: normalising is 1/sqrt(N)
  // (random_vectors.hpp has_deterministic_norm; dist_multivector.hpp:358-362).
  const double scale = normalize ? 1.0 / std::sqrt(static_cast<double>(m->N)) : 1.0;
  const int blocks = std::max(1, std::min(sm_count() * 8, (m->n + 7) / 8));
  if (m->dtype == VBG_C128)
    set_random_kernel<cplx><<<blocks, 256, 0, s>>>(m->n, m->bsz.as<int>(), m->scal_off.as<int64_t>(), k, ld, seed,
                                                    scale, static_cast<cplx*>(X));
  else
    set_random_kernel<double><<<blocks, 256, 0, s>>>(m->n, m->bsz.as<int>(), m->scal_off.as<int64_t>(), k, ld,
                                                      seed, scale, static_cast<double*>(X));
  VBG_CUDA(cudaGetLastError());
  return 0;
}

}  // extern "C"
