// Matrix handles: construction, structure metadata, value transfer and the
// element-wise matrix algebra (scale, shift, add_diagonal, conjugate, block
// norms, duplicate).
//
// Structure follows the reference's serial DistGraph
// (vbcsr/core/dist_graph.hpp:167-312): one block row per block, each row's
// columns sorted ascending (:299), duplicates kept; the value layout is the
// reference's get_values() slot order (vbcsr/core/block_csr.hpp:1202-1248).
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <string>

#include "vbg_internal.cuh"

namespace vbg {

static thread_local std::string g_last_error;

void set_error(const std::string& msg) { g_last_error = msg; }
int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}
int cuda_fail(cudaError_t e, const char* what) {
  g_last_error = std::string(what) + ": " + cudaGetErrorString(e);
  return VBG_E_CUDA;
}

int current_device() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) {
    (void)cudaGetLastError();
    dev = 0;
  }
  return dev < kMaxDevices ? dev : kMaxDevices - 1;
}

int sm_count() {
  static int cached[kMaxDevices] = {};
  const int dev = current_device();
  if (cached[dev] <= 0) {
    int v = 0;
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0) v = 148;
    cached[dev] = v;
  }
  return cached[dev];
}

// Builds host-side structure: per-row sorted columns, slot value offsets,
// scalar offsets, kind.  sort_perm_out (optional) receives, for each sorted
// slot, the index of the input slot it came from.
int build_structure(vbg_matrix* m, int n, const int* bsz, const int* row_ptr, const int* col_ind,
                    std::vector<int64_t>* sort_perm_out) {
  VBG_CHECK(n >= 0, VBG_E_ARG, "negative block row count");
  VBG_CHECK(n == 0 || (bsz && row_ptr), VBG_E_ARG, "null structure arrays");
  VBG_CHECK(n == 0 || row_ptr[0] == 0, VBG_E_ARG, "row_ptr must start at 0");
  for (int i = 0; i < n; ++i) {
    VBG_CHECK(row_ptr[i + 1] >= row_ptr[i], VBG_E_ARG, "row_ptr not monotone");
    VBG_CHECK(bsz[i] >= 1, VBG_E_ARG, "block sizes must be >= 1");
  }
  const int64_t nnzb = n ? row_ptr[n] : 0;
  VBG_CHECK(nnzb == 0 || col_ind, VBG_E_ARG, "null col_ind");
  VBG_CHECK(nnzb <= INT32_MAX, VBG_E_ARG, "more than 2^31 blocks");
  m->n = n;
  m->nnzb = nnzb;
  m->h_bsz.assign(bsz, bsz + n);
  m->h_row_ptr.assign(row_ptr, row_ptr + n + 1);
  if (n == 0) m->h_row_ptr.assign(1, 0);
  m->h_col_ind.resize(nnzb);
  if (sort_perm_out) sort_perm_out->resize(nnzb);
  std::vector<int> idx;
  for (int i = 0; i < n; ++i) {
    const int s0 = row_ptr[i], s1 = row_ptr[i + 1];
    idx.resize(s1 - s0);
    std::iota(idx.begin(), idx.end(), s0);
    bool sorted = true;
    for (int s = s0; s < s1; ++s) {
      VBG_CHECK(col_ind[s] >= 0 && col_ind[s] < n, VBG_E_ARG,
                "column index out of range in row " + std::to_string(i));
      if (s > s0 && col_ind[s] < col_ind[s - 1]) sorted = false;
    }
    if (!sorted)
      std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) { return col_ind[a] < col_ind[b]; });
    for (int s = s0; s < s1; ++s) {
      m->h_col_ind[s] = col_ind[idx[s - s0]];
      if (sort_perm_out) (*sort_perm_out)[s] = idx[s - s0];
    }
  }
  m->host_struct = true;
  m->dup_cols = false;
  for (int i = 0; i < n && !m->dup_cols; ++i)
    for (int sl = m->h_row_ptr[i] + 1; sl < m->h_row_ptr[i + 1]; ++sl)
      if (m->h_col_ind[sl] == m->h_col_ind[sl - 1]) {
        m->dup_cols = true;
        break;
      }
  m->h_scal_off.assign(n + 1, 0);
  for (int i = 0; i < n; ++i) m->h_scal_off[i + 1] = m->h_scal_off[i] + bsz[i];
  m->N = m->h_scal_off[n];
  m->h_blk_off.assign(nnzb + 1, 0);
  for (int i = 0; i < n; ++i)
    for (int s = m->h_row_ptr[i]; s < m->h_row_ptr[i + 1]; ++s)
      m->h_blk_off[s + 1] = m->h_blk_off[s] + (int64_t)bsz[i] * bsz[m->h_col_ind[s]];
  m->nnz = m->h_blk_off[nnzb];
  int mn = n ? bsz[0] : 0, mx = 0;
  for (int i = 0; i < n; ++i) {
    mn = std::min(mn, bsz[i]);
    mx = std::max(mx, bsz[i]);
  }
  m->min_bs = mn;
  m->max_bs = mx;
  // block_csr.hpp:2791-2797: max <= 1 -> CSR, uniform -> BSR, else VBCSR.
  m->kind = (mx <= 1) ? VBG_KIND_CSR : (mn == mx ? VBG_KIND_BSR : VBG_KIND_VBCSR);
  return 0;
}

// Row order used by the apply kernels: rows grouped by block-size class,
// stable so that rows of one class keep their matrix order.
static void class_order(vbg_matrix* m, std::vector<int>& perm) {
  perm.resize(m->n);
  std::iota(perm.begin(), perm.end(), 0);
  std::stable_sort(perm.begin(), perm.end(), [&](int a, int b) { return m->h_bsz[a] < m->h_bsz[b]; });
  m->class_segs.clear();
  for (int w = 0; w < m->n; ++w) {
    const int r = m->h_bsz[perm[w]];
    if (m->class_segs.empty() || m->class_segs.back().r != r) m->class_segs.push_back({r, w, w + 1});
    else m->class_segs.back().w1 = w + 1;
  }
}

template <typename T>
static int upload(DevBuf& buf, const std::vector<T>& v, cudaStream_t s) {
  int rc = buf.ensure(std::max<size_t>(v.size() * sizeof(T), 16));
  if (rc) return rc;
  if (!v.empty()) VBG_CUDA(cudaMemcpyAsync(buf.p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s));
  return 0;
}

int upload_structure(vbg_matrix* m, cudaStream_t s) {
  int rc;
  if ((rc = upload(m->row_ptr, m->h_row_ptr, s))) return rc;
  if ((rc = upload(m->col_ind, m->h_col_ind, s))) return rc;
  if ((rc = upload(m->bsz, m->h_bsz, s))) return rc;
  if ((rc = upload(m->scal_off, m->h_scal_off, s))) return rc;
  if ((rc = upload(m->blk_off, m->h_blk_off, s))) return rc;
  // per-slot gather metadata of the pipelined multivector apply: the first
  // scalar row of the block column and (block rows << 8 | block columns),
  // both modulo their field widths (that kernel only runs when they fit)
  std::vector<int> meta(2 * (size_t)m->nnzb);
  for (int i = 0; i < m->n; ++i)
    for (int sl = m->h_row_ptr[i]; sl < m->h_row_ptr[i + 1]; ++sl) {
      const int col = m->h_col_ind[sl];
      meta[2 * (size_t)sl] = static_cast<int>(static_cast<uint32_t>(m->h_scal_off[col]));
      meta[2 * (size_t)sl + 1] = static_cast<int>(((static_cast<uint32_t>(m->h_bsz[i]) & 0xffu) << 8) |
                                                  (static_cast<uint32_t>(m->h_bsz[col]) & 0xffu));
    }
  if ((rc = upload(m->slot_meta, meta, s))) return rc;
  std::vector<int> diag(m->n, -1);
  for (int i = 0; i < m->n; ++i)
    for (int sl = m->h_row_ptr[i]; sl < m->h_row_ptr[i + 1]; ++sl)
      if (m->h_col_ind[sl] == i) {
        diag[i] = sl;
        break;
      }
  if ((rc = upload(m->diag_slot, diag, s))) return rc;
  std::vector<int> perm;
  class_order(m, perm);
  if ((rc = upload(m->row_perm, perm, s))) return rc;
  // Pageable-memory copies above complete before returning to the host, but
  // the vectors are locals: make sure the stream consumed them.
  VBG_CUDA(cudaStreamSynchronize(s));
  m->invalidate_structure();
  return 0;
}

// ------------------------------------------------------------ kernels

__global__ void to_f32_kernel(const double* __restrict__ a, float* __restrict__ b, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    b[i] = (float)a[i];
}

// Checks a structure given in device memory before anything indexes with it:
// flags[0] row pointers (start at 0, monotone, end at nnzb), flags[1] a
// column outside [0, n), flags[2] columns not ascending within a row,
// flags[3] a column repeated within a row.  A row with bad pointers is not
// read.  A warp per row.
__global__ void check_structure_kernel(int n, int64_t nnzb, const int* __restrict__ rp, const int* __restrict__ ci,
                                       int* __restrict__ flags) {
  const int lane = threadIdx.x & 31;
  const int warps = gridDim.x * (blockDim.x >> 5);
  if (blockIdx.x == 0 && threadIdx.x == 0 && (rp[0] != 0 || (int64_t)rp[n] != nnzb)) atomicOr(flags, 1);
  for (int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); i < n; i += warps) {
    const int s0 = rp[i], s1 = rp[i + 1];
    if (s0 < 0 || s1 < s0 || (int64_t)s1 > nnzb) {
      if (lane == 0) atomicOr(flags, 1);
      continue;
    }
    for (int e = s0 + lane; e < s1; e += 32) {
      const int j = ci[e];
      if (j < 0 || j >= n) atomicOr(flags + 1, 1);
      if (e > s0) {
        const int jp = ci[e - 1];
        if (j < jp) atomicOr(flags + 2, 1);
        if (j == jp) atomicOr(flags + 3, 1);
      }
    }
  }
}

static int grid_for(int64_t n, int threads = 256) {
  int64_t g = (n + threads - 1) / threads;
  const int64_t cap = (int64_t)sm_count() * 16;
  if (g > cap) g = cap;
  if (g < 1) g = 1;
  return (int)g;
}

int ensure_vals32(const vbg_matrix* cm, cudaStream_t s) {
  auto* m = const_cast<vbg_matrix*>(cm);
  if (m->vals32_valid) return 0;
  VBG_CHECK(m->dtype == VBG_F64, VBG_E_STATE, "FP32 shadow is only defined for real FP64 matrices");
  int rc = m->vals32.ensure(std::max<int64_t>(m->nnz, 1) * sizeof(float));
  if (rc) return rc;
  if (m->nnz) to_f32_kernel<<<grid_for(m->nnz), 256, 0, s>>>(m->vals.as<double>(), m->vals32.as<float>(), m->nnz);
  VBG_CUDA(cudaGetLastError());
  m->vals32_valid = true;
  return 0;
}

int ensure_spans(const vbg_matrix* cm, int cap, cudaStream_t s) {
  auto* m = const_cast<vbg_matrix*>(cm);
  if (m->span_cap == cap) return 0;
  {
    const int rc0 = ensure_host_structure(m, s);
    if (rc0) return rc0;
  }
  VBG_CHECK(cap >= m->max_bs && cap < 256, VBG_E_STATE, "span cap must hold the largest block");
  std::vector<int> sp, sptr(m->n + 1, 0);
  std::vector<int64_t> ko, ko32;  // kernel-layout value offset of each span (value type, FP32)
  sp.reserve(4 * (size_t)m->nnzb);
  int64_t count = 0, off = 0, off32 = 0;
  const int es = (int)elem_size(m->dtype);
  for (int i = 0; i < m->n; ++i) {
    const int r = m->h_bsz[i];
    const int rp = kernel_layout_rows(r, es), rp32 = kernel_layout_rows(r, 4);
    int k = m->h_row_ptr[i];
    const int k1 = m->h_row_ptr[i + 1];
    while (k < k1) {
      const int s0 = k;
      int col = m->h_col_ind[k];
      int rows = m->h_bsz[col];
      ++k;
      while (k < k1 && m->h_col_ind[k] == col + 1 && rows + m->h_bsz[col + 1] <= cap) {
        ++col;
        rows += m->h_bsz[col];
        ++k;
      }
      const int64_t o = off, o32 = off32;
      sp.push_back(static_cast<int>(m->h_scal_off[m->h_col_ind[s0]]));
      sp.push_back(rows | (r << 8));
      sp.push_back(static_cast<int>(o & 0xffffffff));
      sp.push_back(static_cast<int>(o >> 32));
      ko32.push_back(o32);
      off += (int64_t)rows * rp;
      off32 += (int64_t)rows * rp32;
      ++count;
    }
    sptr[i + 1] = static_cast<int>(count);
  }
  int rc;
  if ((rc = upload(m->spans, sp, s))) return rc;
  if ((rc = upload(m->span_koff32, ko32, s))) return rc;
  if ((rc = upload(m->row_sptr, sptr, s))) return rc;
  m->h_span_x.resize(count);
  m->h_span_w.resize(count);
  for (int64_t e = 0; e < count; ++e) {
    m->h_span_x[e] = sp[4 * e];
    m->h_span_w[e] = static_cast<unsigned char>(sp[4 * e + 1] & 0xff);
  }
  m->h_row_sptr.swap(sptr);
  m->nspans = count;
  m->span_cap = cap;
  m->tile_plans.clear();  // the plans index spans
  m->chain_plans.clear();
  m->tuned.clear();
  return 0;
}

// One thread per slot: block (r x c, row-major at blk_off) -> c columns of
// kernel_layout_rows(r) scalars at koff, zero padded.
template <typename Tin, typename Tout>
__global__ void kernel_layout_kernel(const Tin* __restrict__ in, const int64_t* __restrict__ blk_off,
                                     const int2* __restrict__ meta, const int64_t* __restrict__ koff, int64_t nnzb,
                                     Tout* __restrict__ out) {
  for (int64_t sl = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; sl < nnzb;
       sl += (int64_t)gridDim.x * blockDim.x) {
    const int rc = meta[sl].y;
    const int r = (rc >> 8) & 0xff, c = rc & 0xff;
    const int rp = kernel_layout_rows(r, (int)sizeof(Tout));
    const Tin* b = in + blk_off[sl];
    Tout* o = out + koff[sl];
    for (int q = 0; q < c; ++q)
      for (int i = 0; i < rp; ++i) o[q * rp + i] = i < r ? static_cast<Tout>(b[i * c + q]) : Tout{};
  }
}

template <>
__global__ void kernel_layout_kernel<cplx, cplx>(const cplx* __restrict__ in, const int64_t* __restrict__ blk_off,
                                                 const int2* __restrict__ meta, const int64_t* __restrict__ koff,
                                                 int64_t nnzb, cplx* __restrict__ out) {
  for (int64_t sl = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; sl < nnzb;
       sl += (int64_t)gridDim.x * blockDim.x) {
    const int rc = meta[sl].y;
    const int r = (rc >> 8) & 0xff, c = rc & 0xff;
    const cplx* b = in + blk_off[sl];
    cplx* o = out + koff[sl];
    for (int q = 0; q < c; ++q)
      for (int i = 0; i < r; ++i) o[q * r + i] = b[i * c + q];
  }
}

int ensure_kernel_layout(const vbg_matrix* cm, bool f32, cudaStream_t s) {
  auto* m = const_cast<vbg_matrix*>(cm);
  if (f32 ? m->valsK32_valid : m->valsK_valid) return 0;
  VBG_CHECK(m->max_bs <= 8, VBG_E_STATE, "kernel layout needs blocks of at most 8 x 8");
  VBG_CHECK(!f32 || m->dtype == VBG_F64, VBG_E_STATE, "FP32 shadow is only defined for real FP64 matrices");
  int rc;
  if (!m->koff_valid) {
    if ((rc = ensure_host_structure(m, s))) return rc;
    // offsets for the value type and for FP32
    const int es = (int)elem_size(m->dtype);
    std::vector<int64_t> off(m->nnzb + 1, 0), off32(m->nnzb + 1, 0);
    for (int i = 0; i < m->n; ++i)
      for (int sl = m->h_row_ptr[i]; sl < m->h_row_ptr[i + 1]; ++sl) {
        const int r = m->h_bsz[i], c = m->h_bsz[m->h_col_ind[sl]];
        off[sl + 1] = off[sl] + (int64_t)c * kernel_layout_rows(r, es);
        off32[sl + 1] = off32[sl] + (int64_t)c * kernel_layout_rows(r, 4);
      }
    // pageable sources: each copy has read its source when the call returns
    if ((rc = upload(m->koff, off, s))) return rc;
    if ((rc = upload(m->koff32, off32, s))) return rc;
    m->koff_total = off[m->nnzb];
    m->koff32_total = off32[m->nnzb];
    m->koff_valid = true;
  }
  const int64_t total = f32 ? m->koff32_total : m->koff_total;
  const int2* meta = m->slot_meta.as<int2>();
  if (f32) {
    if ((rc = m->valsK32.ensure(std::max<int64_t>(total, 4) * sizeof(float)))) return rc;
    if (m->nnzb)
      kernel_layout_kernel<double, float><<<grid_for(m->nnzb), 256, 0, s>>>(
          m->vals.as<double>(), m->blk_off.as<int64_t>(), meta, m->koff32.as<int64_t>(), m->nnzb,
          m->valsK32.as<float>());
    VBG_CUDA(cudaGetLastError());
    m->valsK32_valid = true;
  } else {
    if ((rc = m->valsK.ensure(std::max<int64_t>(total, 1) * elem_size(m->dtype)))) return rc;
    if (m->nnzb) {
      if (m->dtype == VBG_C128)
        kernel_layout_kernel<cplx, cplx><<<grid_for(m->nnzb), 256, 0, s>>>(
            m->vals.as<cplx>(), m->blk_off.as<int64_t>(), meta, m->koff.as<int64_t>(), m->nnzb, m->valsK.as<cplx>());
      else
        kernel_layout_kernel<double, double><<<grid_for(m->nnzb), 256, 0, s>>>(
            m->vals.as<double>(), m->blk_off.as<int64_t>(), meta, m->koff.as<int64_t>(), m->nnzb,
            m->valsK.as<double>());
    }
    VBG_CUDA(cudaGetLastError());
    m->valsK_valid = true;
  }
  // later applies may run on other streams
  VBG_CUDA(cudaStreamSynchronize(s));
  return 0;
}

// Column-major view for the adjoint: for each block column j the slots (i, j)
// in increasing row order (the reference's column-incoming plan,
// vbcsr/core/detail/backend/vbcsr_backend.hpp:543-625).
int ensure_csc(const vbg_matrix* cm, cudaStream_t s) { return build_csc_dev(cm, s); }

int ensure_scratch(const vbg_matrix* cm, int grid) {
  auto* m = const_cast<vbg_matrix*>(cm);
  int rc = m->partials.ensure((size_t)grid * 2 * sizeof(double));
  if (rc) return rc;
  if (!m->counter.p) {
    rc = m->counter.ensure(256);
    if (rc) return rc;
    VBG_CUDA(cudaMemset(m->counter.p, 0, 256));
  }
  return 0;
}

template <typename T>
__global__ void scale_kernel(T* v, int64_t n, double re, double im);
template <>
__global__ void scale_kernel<double>(double* v, int64_t n, double re, double) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    v[i] *= re;
}
template <>
__global__ void scale_kernel<cplx>(cplx* v, int64_t n, double re, double im) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const cplx a = v[i];
    v[i] = {a.re * re - a.im * im, a.re * im + a.im * re};
  }
}

__global__ void conj_kernel(cplx* v, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    v[i].im = -v[i].im;
}

// A_ii += alpha (shift) or A_ii += v[scal_off[i] + t] (add_diagonal): one
// thread per block row, on the row's diagonal block (block_csr.hpp:1289-1370).
template <typename T>
__global__ void diag_kernel(T* vals, const int* __restrict__ diag_slot, const int64_t* __restrict__ blk_off,
                            const int* __restrict__ bsz, const int64_t* __restrict__ scal_off, int n, double re,
                            double im, const T* __restrict__ v) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int s = diag_slot[i];
    if (s < 0) continue;
    const int r = bsz[i];
    T* b = vals + blk_off[s];
    for (int t = 0; t < r; ++t) {
      if constexpr (sizeof(T) == sizeof(cplx)) {
        cplx add = v ? reinterpret_cast<const cplx*>(v)[scal_off[i] + t] : cplx{re, im};
        cplx* e = reinterpret_cast<cplx*>(b) + t * r + t;
        e->re += add.re;
        e->im += add.im;
      } else {
        const double add = v ? reinterpret_cast<const double*>(v)[scal_off[i] + t] : re;
        reinterpret_cast<double*>(b)[t * r + t] += add;
      }
    }
  }
}

// Frobenius norm per block: sum of squares in element order, each square
// rounded before the add exactly as the reference source writes it
// (block_csr.hpp:2487-2502, block_squared_magnitude at
// ops/spmm/common.hpp:184-191), one thread per block.
template <typename T>
__global__ void norms_kernel(const T* __restrict__ vals, const int64_t* __restrict__ blk_off, int64_t nnzb,
                             double* __restrict__ out) {
  for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < nnzb; s += (int64_t)gridDim.x * blockDim.x) {
    const int64_t a = blk_off[s], b = blk_off[s + 1];
    double sum = 0.0;
    for (int64_t k = a; k < b; ++k) {
      if constexpr (sizeof(T) == sizeof(cplx)) {
        const cplx z = reinterpret_cast<const cplx*>(vals)[k];
        sum = __dadd_rn(sum, fma(z.re, z.re, __dmul_rn(z.im, z.im)));
      } else {
        const double x = reinterpret_cast<const double*>(vals)[k];
        sum = __dadd_rn(sum, __dmul_rn(x, x));
      }
    }
    out[s] = sqrt(sum);
  }
}

int block_norms_dev(const vbg_matrix* m, double* out, cudaStream_t s) {
  if (m->nnzb == 0) return 0;
  if (m->dtype == VBG_C128)
    norms_kernel<cplx><<<grid_for(m->nnzb), 256, 0, s>>>(m->vals.as<cplx>(), m->blk_off.as<int64_t>(), m->nnzb, out);
  else
    norms_kernel<double><<<grid_for(m->nnzb), 256, 0, s>>>(m->vals.as<double>(), m->blk_off.as<int64_t>(), m->nnzb, out);
  VBG_CUDA(cudaGetLastError());
  return 0;
}

// Fixed-order FP64 reductions over a matrix (trace, Frobenius norm): a
// fixed grid writes two partial sums per CTA, one CTA adds them in order.
constexpr int kReduceCtas = 256;

// A two-value sum over the 256 threads of a block (fixed order); thread 0
// gets it.
__device__ void block_sum2_256(double& a, double& b) {
  __shared__ double sa[256], sb[256];
  sa[threadIdx.x] = a;
  sb[threadIdx.x] = b;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) {
      sa[threadIdx.x] += sa[threadIdx.x + w];
      sb[threadIdx.x] += sb[threadIdx.x + w];
    }
    __syncthreads();
  }
  a = sa[0];
  b = sb[0];
}

template <typename T>
__global__ void trace_partials(const T* __restrict__ vals, const int* __restrict__ diag_slot,
                               const int64_t* __restrict__ blk_off, const int* __restrict__ bsz, int n,
                               double* __restrict__ part) {
  double re = 0.0, im = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int sl = diag_slot[i];
    if (sl < 0) continue;
    const int r = bsz[i];
    const T* b = vals + blk_off[sl];
    for (int t = 0; t < r; ++t) {
      if constexpr (sizeof(T) == sizeof(cplx)) {
        const cplx e = reinterpret_cast<const cplx*>(b)[t * r + t];
        re += e.re;
        im += e.im;
      } else {
        re += reinterpret_cast<const double*>(b)[t * r + t];
      }
    }
  }
  block_sum2_256(re, im);
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = re;
    part[2 * blockIdx.x + 1] = im;
  }
}

__global__ void sumsq_partials(const double* __restrict__ v, int64_t n, double* __restrict__ part) {
  double a = 0.0, b = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    a = fma(v[i], v[i], a);
  block_sum2_256(a, b);
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = a;
    part[2 * blockIdx.x + 1] = 0.0;
  }
}

// out[0..1] = the sums of the partials (sqrt of the first when `root`).
__global__ void sum_partials(const double* __restrict__ part, int nparts, double* __restrict__ out, bool root) {
  double a = 0.0, b = 0.0;
  for (int k = threadIdx.x; k < nparts; k += blockDim.x) {
    a += part[2 * k];
    b += part[2 * k + 1];
  }
  block_sum2_256(a, b);
  if (threadIdx.x == 0) {
    out[0] = root ? sqrt(a) : a;
    out[1] = b;
  }
}

// The per-CTA partials of the reductions, in the matrix's reduction scratch.
static int reduction_scratch(const vbg_matrix* m, double** part) {
  int rc = ensure_scratch(m, kReduceCtas);
  if (rc) return rc;
  *part = m->partials.as<double>();
  return 0;
}

}  // namespace vbg

using namespace vbg;

extern "C" {

int vbg_version(void) { return 1; }
const char* vbg_last_error(void) { return g_last_error.c_str(); }
int vbg_device_count(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) {
    (void)cudaGetLastError();
    return 0;
  }
  return n;
}

int vbg_matrix_create(vbg_matrix** out, int dtype, int n, const int* bsz, const int* row_ptr, const int* col_ind,
                      const void* values, void* stream) {
  VBG_CHECK(out, VBG_E_ARG, "out is null");
  VBG_CHECK(dtype == VBG_F64 || dtype == VBG_C128, VBG_E_ARG, "unknown dtype");
  *out = nullptr;
  if (vbg_device_count() == 0) return fail(VBG_E_CUDA, "no CUDA device is visible");
  auto m = std::make_unique<vbg_matrix>();
  m->dtype = dtype;
  cudaGetDevice(&m->device);
  int rc = build_structure(m.get(), n, bsz, row_ptr, col_ind, nullptr);
  if (rc) return rc;
  cudaStream_t s = as_stream(stream);
  if ((rc = upload_structure(m.get(), s))) return rc;
  const size_t vb = std::max<int64_t>(m->nnz, 1) * elem_size(dtype);
  if ((rc = m->vals.ensure(vb))) return rc;
  if (values && m->nnz)
    VBG_CUDA(cudaMemcpyAsync(m->vals.p, values, m->nnz * elem_size(dtype), cudaMemcpyHostToDevice, s));
  else
    VBG_CUDA(cudaMemsetAsync(m->vals.p, 0, vb, s));
  VBG_CUDA(cudaStreamSynchronize(s));
  *out = m.release();
  return 0;
}

int vbg_matrix_create_device(vbg_matrix** out, int dtype, int n, const int* bsz, int64_t nnzb,
                             const int* row_ptr_dev, const int* col_ind_dev, const void* values_dev, void* stream) {
  VBG_CHECK(out, VBG_E_ARG, "out is null");
  VBG_CHECK(dtype == VBG_F64 || dtype == VBG_C128, VBG_E_ARG, "unknown dtype");
  VBG_CHECK(n >= 0 && nnzb >= 0 && nnzb <= INT32_MAX, VBG_E_ARG, "invalid block row or block count");
  VBG_CHECK(n == 0 || (bsz && row_ptr_dev), VBG_E_ARG, "null structure arrays");
  VBG_CHECK(nnzb == 0 || col_ind_dev, VBG_E_ARG, "null col_ind");
  *out = nullptr;
  if (vbg_device_count() == 0) return fail(VBG_E_CUDA, "no CUDA device is visible");
  for (int i = 0; i < n; ++i) VBG_CHECK(bsz[i] >= 1, VBG_E_ARG, "block sizes must be >= 1");
  auto m = std::make_unique<vbg_matrix>();
  m->dtype = dtype;
  cudaGetDevice(&m->device);
  cudaStream_t s = as_stream(stream);
  // the per-row part from the block sizes (host, O(n))
  m->n = n;
  m->nnzb = nnzb;
  m->h_bsz.assign(bsz, bsz + n);
  m->h_scal_off.assign(n + 1, 0);
  for (int i = 0; i < n; ++i) m->h_scal_off[i + 1] = m->h_scal_off[i] + bsz[i];
  m->N = m->h_scal_off[n];
  int mn = n ? bsz[0] : 0, mx = 0;
  for (int i = 0; i < n; ++i) {
    mn = std::min(mn, bsz[i]);
    mx = std::max(mx, bsz[i]);
  }
  m->min_bs = mn;
  m->max_bs = mx;
  m->kind = (mx <= 1) ? VBG_KIND_CSR : (mn == mx ? VBG_KIND_BSR : VBG_KIND_VBCSR);
  std::vector<int> perm;
  class_order(m.get(), perm);
  int rc;
  if ((rc = upload(m->bsz, m->h_bsz, s))) return rc;
  if ((rc = upload(m->scal_off, m->h_scal_off, s))) return rc;
  if ((rc = upload(m->row_perm, perm, s))) return rc;
  // the per-slot part from the caller's device arrays
  if ((rc = m->row_ptr.ensure((n + 1) * sizeof(int), s))) return rc;
  if ((rc = m->col_ind.ensure(std::max<int64_t>(nnzb, 1) * sizeof(int), s))) return rc;
  if (n) VBG_CUDA(cudaMemcpyAsync(m->row_ptr.p, row_ptr_dev, (n + 1) * sizeof(int), cudaMemcpyDeviceToDevice, s));
  else VBG_CUDA(cudaMemsetAsync(m->row_ptr.p, 0, sizeof(int), s));
  if (nnzb) VBG_CUDA(cudaMemcpyAsync(m->col_ind.p, col_ind_dev, nnzb * sizeof(int), cudaMemcpyDeviceToDevice, s));
  DevBuf flags(s);
  if ((rc = flags.ensure(4 * sizeof(int)))) return rc;
  VBG_CUDA(cudaMemsetAsync(flags.p, 0, 4 * sizeof(int), s));
  if (n) {
    check_structure_kernel<<<std::max(1, std::min((n + 7) / 8, sm_count() * 16)), 256, 0, s>>>(
        n, nnzb, m->row_ptr.as<int>(), m->col_ind.as<int>(), flags.as<int>());
    VBG_CUDA(cudaGetLastError());
  }
  int hf[4] = {0, 0, 0, 0};
  VBG_CUDA(cudaMemcpyAsync(hf, flags.p, sizeof(hf), cudaMemcpyDeviceToHost, s));
  VBG_CUDA(cudaStreamSynchronize(s));
  VBG_CHECK(hf[0] == 0, VBG_E_ARG, "row_ptr must start at 0, be monotone and end at nnzb");
  VBG_CHECK(hf[1] == 0, VBG_E_ARG, "column index out of range");
  VBG_CHECK(hf[2] == 0, VBG_E_ARG, "columns must be sorted within each row (device construction does not sort)");
  m->dup_cols = hf[3] != 0;
  m->host_struct = false;  // the host mirrors are read back on first use
  if ((rc = device_slot_structure(m.get(), s))) return rc;
  const size_t vb = std::max<int64_t>(m->nnz, 1) * elem_size(dtype);
  if ((rc = m->vals.ensure(vb))) return rc;
  if (values_dev && m->nnz)
    VBG_CUDA(cudaMemcpyAsync(m->vals.p, values_dev, m->nnz * elem_size(dtype), cudaMemcpyDeviceToDevice, s));
  else
    VBG_CUDA(cudaMemsetAsync(m->vals.p, 0, vb, s));
  VBG_CUDA(cudaStreamSynchronize(s));
  m->invalidate_structure();
  *out = m.release();
  return 0;
}

int vbg_matrix_destroy(vbg_matrix* m) {
  delete m;
  return 0;
}

int vbg_matrix_duplicate(const vbg_matrix* m, vbg_matrix** out, void* stream) {
  VBG_CHECK(m && out, VBG_E_ARG, "null argument");
  auto d = std::make_unique<vbg_matrix>();
  d->dtype = m->dtype;
  d->device = m->device;
  cudaStream_t s = as_stream(stream);
  int rc = ensure_host_structure(m, s);
  if (rc) return rc;
  if ((rc = build_structure(d.get(), m->n, m->h_bsz.data(), m->h_row_ptr.data(), m->h_col_ind.data(), nullptr)))
    return rc;
  if ((rc = upload_structure(d.get(), s))) return rc;
  if ((rc = d->vals.ensure(std::max<int64_t>(m->nnz, 1) * elem_size(m->dtype)))) return rc;
  if (m->nnz) VBG_CUDA(cudaMemcpyAsync(d->vals.p, m->vals.p, m->nnz * elem_size(m->dtype), cudaMemcpyDeviceToDevice, s));
  *out = d.release();
  return 0;
}

int vbg_matrix_info(const vbg_matrix* m, int* dtype, int* n, int64_t* nnzb, int64_t* nnz, int64_t* N, int* kind) {
  VBG_CHECK(m, VBG_E_ARG, "null matrix");
  if (dtype) *dtype = m->dtype;
  if (n) *n = m->n;
  if (nnzb) *nnzb = m->nnzb;
  if (nnz) *nnz = m->nnz;
  if (N) *N = m->N;
  if (kind) *kind = m->kind;
  return 0;
}

int vbg_matrix_get_structure(const vbg_matrix* m, int* row_ptr, int* col_ind, int* block_sizes) {
  VBG_CHECK(m, VBG_E_ARG, "null matrix");
  int rc = ensure_host_structure(m, nullptr);
  if (rc) return rc;
  if (row_ptr) std::memcpy(row_ptr, m->h_row_ptr.data(), (m->n + 1) * sizeof(int));
  if (col_ind && m->nnzb) std::memcpy(col_ind, m->h_col_ind.data(), m->nnzb * sizeof(int));
  if (block_sizes && m->n) std::memcpy(block_sizes, m->h_bsz.data(), m->n * sizeof(int));
  return 0;
}

int vbg_matrix_get_values(const vbg_matrix* m, void* values, void* stream) {
  VBG_CHECK(m && (values || !m->nnz), VBG_E_ARG, "null argument");
  if (!m->nnz) return 0;
  cudaStream_t s = as_stream(stream);
  VBG_CUDA(cudaMemcpyAsync(values, m->vals.p, m->nnz * elem_size(m->dtype), cudaMemcpyDeviceToHost, s));
  VBG_CUDA(cudaStreamSynchronize(s));
  return 0;
}

int vbg_matrix_set_values(vbg_matrix* m, const void* values, void* stream) {
  VBG_CHECK(m && (values || !m->nnz), VBG_E_ARG, "null argument");
  if (!m->nnz) return 0;
  cudaStream_t s = as_stream(stream);
  VBG_CUDA(cudaMemcpyAsync(m->vals.p, values, m->nnz * elem_size(m->dtype), cudaMemcpyHostToDevice, s));
  VBG_CUDA(cudaStreamSynchronize(s));
  m->invalidate_values();
  return 0;
}

int vbg_matrix_set_values_device(vbg_matrix* m, const void* values_dev, void* stream) {
  VBG_CHECK(m && (values_dev || !m->nnz), VBG_E_ARG, "null argument");
  if (!m->nnz) return 0;
  VBG_CUDA(cudaMemcpyAsync(m->vals.p, values_dev, m->nnz * elem_size(m->dtype), cudaMemcpyDeviceToDevice,
                           as_stream(stream)));
  m->invalidate_values();
  return 0;
}

int vbg_matrix_device_values(const vbg_matrix* m, void** values, const int64_t** offs) {
  VBG_CHECK(m, VBG_E_ARG, "null matrix");
  if (values) *values = m->vals.p;
  if (offs) *offs = m->blk_off.as<int64_t>();
  return 0;
}

int vbg_matrix_block_norms(const vbg_matrix* m, double* norms_dev, void* stream) {
  VBG_CHECK(m && (norms_dev || !m->nnzb), VBG_E_ARG, "null argument");
  return block_norms_dev(m, norms_dev, as_stream(stream));
}

int vbg_matrix_scale(vbg_matrix* m, double re, double im, void* stream) {
  VBG_CHECK(m, VBG_E_ARG, "null matrix");
  if (!m->nnz) return 0;
  cudaStream_t s = as_stream(stream);
  if (m->dtype == VBG_C128)
    scale_kernel<cplx><<<grid_for(m->nnz), 256, 0, s>>>(m->vals.as<cplx>(), m->nnz, re, im);
  else
    scale_kernel<double><<<grid_for(m->nnz), 256, 0, s>>>(m->vals.as<double>(), m->nnz, re, im);
  VBG_CUDA(cudaGetLastError());
  m->invalidate_values();
  return 0;
}

int vbg_matrix_conjugate(vbg_matrix* m, void* stream) {
  VBG_CHECK(m, VBG_E_ARG, "null matrix");
  if (m->dtype != VBG_C128 || !m->nnz) return 0;
  conj_kernel<<<grid_for(m->nnz), 256, 0, as_stream(stream)>>>(m->vals.as<cplx>(), m->nnz);
  VBG_CUDA(cudaGetLastError());
  m->invalidate_values();
  return 0;
}

static int diag_op(vbg_matrix* m, double re, double im, const void* v, void* stream) {
  VBG_CHECK(m, VBG_E_ARG, "null matrix");
  if (!m->n) return 0;
  cudaStream_t s = as_stream(stream);
  if (m->dtype == VBG_C128)
    diag_kernel<cplx><<<grid_for(m->n), 256, 0, s>>>(m->vals.as<cplx>(), m->diag_slot.as<int>(),
                                                       m->blk_off.as<int64_t>(), m->bsz.as<int>(),
                                                       m->scal_off.as<int64_t>(), m->n, re, im,
                                                       static_cast<const cplx*>(v));
  else
    diag_kernel<double><<<grid_for(m->n), 256, 0, s>>>(m->vals.as<double>(), m->diag_slot.as<int>(),
                                                         m->blk_off.as<int64_t>(), m->bsz.as<int>(),
                                                         m->scal_off.as<int64_t>(), m->n, re, im,
                                                         static_cast<const double*>(v));
  VBG_CUDA(cudaGetLastError());
  m->invalidate_values();
  return 0;
}

int vbg_matrix_shift(vbg_matrix* m, double re, double im, void* stream) { return diag_op(m, re, im, nullptr, stream); }

int vbg_matrix_trace(const vbg_matrix* m, double* out, void* stream) {
  VBG_CHECK(m && out, VBG_E_ARG, "null argument");
  cudaStream_t s = as_stream(stream);
  double* part = nullptr;
  int rc = reduction_scratch(m, &part);
  if (rc) return rc;
  if (m->dtype == VBG_C128)
    trace_partials<cplx><<<kReduceCtas, 256, 0, s>>>(m->vals.as<cplx>(), m->diag_slot.as<int>(),
                                                     m->blk_off.as<int64_t>(), m->bsz.as<int>(), m->n, part);
  else
    trace_partials<double><<<kReduceCtas, 256, 0, s>>>(m->vals.as<double>(), m->diag_slot.as<int>(),
                                                       m->blk_off.as<int64_t>(), m->bsz.as<int>(), m->n, part);
  VBG_CUDA(cudaGetLastError());
  sum_partials<<<1, 256, 0, s>>>(part, kReduceCtas, out, false);
  VBG_CUDA(cudaGetLastError());
  return 0;
}

int vbg_matrix_norm_fro(const vbg_matrix* m, double* out, void* stream) {
  VBG_CHECK(m && out, VBG_E_ARG, "null argument");
  cudaStream_t s = as_stream(stream);
  double* part = nullptr;
  int rc = reduction_scratch(m, &part);
  if (rc) return rc;
  const int64_t nscal = m->dtype == VBG_C128 ? 2 * m->nnz : m->nnz;  // a complex value is two doubles
  sumsq_partials<<<kReduceCtas, 256, 0, s>>>(m->vals.as<double>(), nscal, part);
  VBG_CUDA(cudaGetLastError());
  sum_partials<<<1, 256, 0, s>>>(part, kReduceCtas, out, true);
  VBG_CUDA(cudaGetLastError());
  return 0;
}
int vbg_matrix_add_diagonal(vbg_matrix* m, const void* v, void* stream) {
  VBG_CHECK(v, VBG_E_ARG, "null vector");
  return diag_op(m, 0, 0, v, stream);
}

}  // extern "C"
