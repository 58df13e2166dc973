// Pattern-restricted outer products (SDDMM) for the gradients of the sparse
// apply: out_ij += alpha * G_i X_j^H over the stored blocks (i, j) of A, with
// G_i the r rows of G at block row i and X_j the c rows of X at block column
// j (k columns each).  For Y = A X and a real loss with dL/dY* = G this is
// dL/dA* restricted to A's pattern, the term a hand-written backward of the
// apply (and of the Chebyshev recurrence built on it) needs; the reference
// has no gradients, so there is no reference routine to mirror.
//
// Layout: `out` has A's value layout (slot order, r x c row-major blocks);
// G and X are row-major multivectors with leading dimension ld (ld = 1: plain
// vectors).  One warp per block row (rows in natural order, grid-stride):
// the warp stages the block row's G rows once and each block's X rows in
// shared memory (blocks up to 8 x 8, up to 32 columns; coalesced copies),
// then lanes own the (o, q) entries of the block and each reduces the k
// products G[o, :] . conj(X[q, :]) from shared memory -- one copy of every
// row instead of one global read per entry that uses it.  A block row's
// slots are written by its warp only, so the read-modify-write of `out`
// needs no atomics.
#include <algorithm>

#include "vbg_internal.cuh"

namespace vbg {

constexpr int kSddmmWarps = 8;
// Staging in shared memory: blocks of up to 8 rows / columns, up to 32
// multivector columns; larger ones read G and X from global memory.
constexpr int kSddmmStageRows = 8;
constexpr int kSddmmStageK = 32;

__device__ __forceinline__ double conj_mul(double g, double x) { return g * x; }
__device__ __forceinline__ cplx conj_mul(cplx g, cplx x) {
  return {fma(g.re, x.re, g.im * x.im), fma(g.im, x.re, -g.re * x.im)};
}
__device__ __forceinline__ double mul_s(double a, double b) { return a * b; }
__device__ __forceinline__ cplx mul_s(cplx a, cplx b) { return {fma(a.re, b.re, -a.im * b.im), fma(a.re, b.im, a.im * b.re)}; }
template <typename T> __device__ __forceinline__ T scalar_from(double re, double im);
template <> __device__ __forceinline__ double scalar_from<double>(double re, double) { return re; }
template <> __device__ __forceinline__ cplx scalar_from<cplx>(double re, double im) { return {re, im}; }

template <typename T>
__global__ void __launch_bounds__(kSddmmWarps * 32)
    sddmm_kernel(int n_rows, const int* __restrict__ row_ptr, const int* __restrict__ col_ind,
                 const int* __restrict__ bsz, const int64_t* __restrict__ scal_off,
                 const int64_t* __restrict__ blk_off, int k, int ld, const T* __restrict__ G,
                 const T* __restrict__ X, double are, double aim, T* __restrict__ out) {
  const int lane = threadIdx.x & 31;
  const T alpha = scalar_from<T>(are, aim);
  // per warp: the block row's G rows and the current block's X rows, each row
  // padded by one scalar (kp = k + 1) so rows start in different banks
  extern __shared__ unsigned char sddmm_smem[];
  const int kp = k + 1;
  const bool staged = k <= kSddmmStageK;
  T* Gs = reinterpret_cast<T*>(sddmm_smem) + (size_t)(threadIdx.x >> 5) * 2 * kSddmmStageRows * (kSddmmStageK + 1);
  T* Xs = Gs + kSddmmStageRows * (kSddmmStageK + 1);
  for (int i = blockIdx.x * kSddmmWarps + (threadIdx.x >> 5); i < n_rows; i += gridDim.x * kSddmmWarps) {
    const int r = bsz[i];
    const T* Gi = G + scal_off[i] * (int64_t)ld;
    const bool g_in = staged && r <= kSddmmStageRows;
    if (g_in) {
      for (int idx = lane; idx < r * k; idx += 32) {
        const int o = idx / k, t = idx - o * k;
        Gs[o * kp + t] = Gi[(int64_t)o * ld + t];
      }
      __syncwarp();
    }
    for (int e = row_ptr[i]; e < row_ptr[i + 1]; ++e) {
      const int j = col_ind[e];
      const int c = bsz[j];
      const T* Xj = X + scal_off[j] * (int64_t)ld;
      T* ob = out + blk_off[e];
      if (g_in && c <= kSddmmStageRows) {
        for (int idx = lane; idx < c * k; idx += 32) {
          const int q = idx / k, t = idx - q * k;
          Xs[q * kp + t] = Xj[(int64_t)q * ld + t];
        }
        __syncwarp();
        for (int p = lane; p < r * c; p += 32) {
          const int o = p / c, q = p - o * c;
          const T* g = Gs + o * kp;
          const T* x = Xs + q * kp;
          T s = zero_s<T>();
          for (int t = 0; t < k; ++t) s = s + conj_mul(g[t], x[t]);
          ob[p] = ob[p] + mul_s(alpha, s);
        }
        __syncwarp();  // Xs is rewritten for the next block
      } else {
        for (int p = lane; p < r * c; p += 32) {
          const int o = p / c, q = p - o * c;
          const T* g = Gi + (int64_t)o * ld;
          const T* x = Xj + (int64_t)q * ld;
          T s = zero_s<T>();
          for (int t = 0; t < k; ++t) s = s + conj_mul(g[t], x[t]);
          ob[p] = ob[p] + mul_s(alpha, s);
        }
      }
    }
    __syncwarp();  // Gs is rewritten for the next row
  }
}

}  // namespace vbg

using namespace vbg;

extern "C" int vbg_sddmm(const vbg_matrix* m, int k, int ld, const void* G, const void* X, double alpha_re,
                         double alpha_im, void* out, void* stream) {
  VBG_CHECK(m, VBG_E_ARG, "null matrix");
  VBG_CHECK(k >= 1 && ld >= k, VBG_E_ARG, "invalid k / ld");
  VBG_CHECK((G && X && out) || m->nnz == 0, VBG_E_ARG, "null argument");
  if (m->n == 0 || m->nnz == 0) return 0;
  cudaStream_t s = as_stream(stream);
  const int grid = std::max(1, std::min((m->n + kSddmmWarps - 1) / kSddmmWarps, sm_count() * 8));
  const size_t es = m->dtype == VBG_C128 ? sizeof(cplx) : sizeof(double);
  const size_t smem = (size_t)kSddmmWarps * 2 * kSddmmStageRows * (kSddmmStageK + 1) * es;
  // the staging needs more than the default 48 KB per CTA (complex values)
  if (m->dtype == VBG_C128)
    VBG_CUDA(cudaFuncSetAttribute(sddmm_kernel<cplx>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  else
    VBG_CUDA(cudaFuncSetAttribute(sddmm_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  if (m->dtype == VBG_C128)
    sddmm_kernel<cplx><<<grid, kSddmmWarps * 32, smem, s>>>(
        m->n, m->row_ptr.as<int>(), m->col_ind.as<int>(), m->bsz.as<int>(), m->scal_off.as<int64_t>(),
        m->blk_off.as<int64_t>(), k, ld, static_cast<const cplx*>(G), static_cast<const cplx*>(X), alpha_re, alpha_im,
        static_cast<cplx*>(out));
  else
    sddmm_kernel<double><<<grid, kSddmmWarps * 32, smem, s>>>(
        m->n, m->row_ptr.as<int>(), m->col_ind.as<int>(), m->bsz.as<int>(), m->scal_off.as<int64_t>(),
        m->blk_off.as<int64_t>(), k, ld, static_cast<const double*>(G), static_cast<const double*>(X), alpha_re,
        alpha_im, static_cast<double*>(out));
  VBG_CUDA(cudaGetLastError());
  return 0;
}
