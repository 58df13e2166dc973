// Structure-changing matrix algebra: axpby (same / subset / union pattern),
// conjugate transpose and the Frobenius block filter.
//
// Reference behaviour replaced:
//   VBCSRAxpbyExecutor::run    vbcsr/core/detail/ops/axpby.hpp:254-420
//   conjugate_transpose        vbcsr/core/detail/ops/transpose.hpp:179
//   BlockSpMat::filter_blocks  vbcsr/core/block_csr.hpp:1399-1528
//
// The structure (row pointers, sorted column lists) is kept on the host as
// well as on the device; pattern merges are done there (O(nnzb) integer
// work), the value movement by one gather kernel on the device.
#include <algorithm>
#include <cstring>
#include <vector>

#include "vbg_internal.cuh"

namespace vbg {

int block_norms_dev(const vbg_matrix* m, double* out, cudaStream_t s);

// out[p] = alpha * A[mapA[p]] (+ beta * B[mapB[p]]), block by block; map -1
// contributes zero.  transpose != 0: A's block is conj-transposed into p.
template <typename T>
__global__ void gather_combine_kernel(int64_t nout, const int64_t* __restrict__ out_off, T* __restrict__ out,
                                      const int* __restrict__ out_row, const int* __restrict__ out_col,
                                      const int* __restrict__ bsz, const T* __restrict__ A,
                                      const int64_t* __restrict__ a_off, const int* __restrict__ mapA, double are,
                                      double aim, const T* __restrict__ B, const int64_t* __restrict__ b_off,
                                      const int* __restrict__ mapB, double bre, double bim, int transpose) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t p = blockIdx.x * (int64_t)(blockDim.x >> 5) + (threadIdx.x >> 5); p < nout; p += warps) {
    const int64_t o0 = out_off[p], len = out_off[p + 1] - o0;
    const int sa = mapA ? mapA[p] : -1;
    const int sb = mapB ? mapB[p] : -1;
    const int rows_out = transpose ? bsz[out_row[p]] : 0, cols_out = transpose ? bsz[out_col[p]] : 1;
    for (int64_t e = lane; e < len; e += 32) {
      T acc = zero_s<T>();
      if (sa >= 0) {
        int64_t ie = e;
        if (transpose) {
          const int64_t q = e / cols_out, t = e - q * cols_out;
          ie = t * rows_out + q;
        }
        T a = A[a_off[sa] + ie];
        if (transpose) a = conj_s(a);
        acc = cmad(are, aim, a, acc);
      }
      if (sb >= 0) acc = cmad(bre, bim, B[b_off[sb] + e], acc);
      out[o0 + e] = acc;
    }
  }
}

// Y <- alpha X + beta Y element by element (same pattern, same slot offsets),
// with the arithmetic of gather_combine_kernel.
template <typename T>
__global__ void axpby_same_kernel(int64_t n, double are, double aim, const T* __restrict__ X, double bre, double bim,
                                  T* __restrict__ Y) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    Y[i] = cmad(bre, bim, Y[i], cmad(are, aim, X[i], zero_s<T>()));
}

// Sets *flag to 1 if a[i] != b[i] for some i < n.
__global__ void differ_kernel(const int* __restrict__ a, const int* __restrict__ b, int64_t n, int* flag) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    if (a[i] != b[i]) {
      *flag = 1;
      return;
    }
}

// Whether Y and X have the same pattern: compared on the host when both
// mirrors are current, else on the device.
static int same_pattern(const vbg_matrix* Y, const vbg_matrix* X, bool* same, cudaStream_t s) {
  *same = false;
  if (Y->nnzb != X->nnzb) return 0;
  if (Y->host_struct && X->host_struct) {
    *same = Y->h_row_ptr == X->h_row_ptr && Y->h_col_ind == X->h_col_ind;
    return 0;
  }
  int rc;
  DevBuf flag(s);
  if ((rc = flag.ensure(sizeof(int)))) return rc;
  VBG_CUDA(cudaMemsetAsync(flag.p, 0, sizeof(int), s));
  const int64_t total = (int64_t)Y->n + 1 + Y->nnzb;
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((total + 255) / 256, sm_count() * 8));
  differ_kernel<<<grid, 256, 0, s>>>(Y->row_ptr.as<int>(), X->row_ptr.as<int>(), Y->n + 1, flag.as<int>());
  if (Y->nnzb)
    differ_kernel<<<grid, 256, 0, s>>>(Y->col_ind.as<int>(), X->col_ind.as<int>(), Y->nnzb, flag.as<int>());
  VBG_CUDA(cudaGetLastError());
  int h = 0;
  VBG_CUDA(cudaMemcpyAsync(&h, flag.p, sizeof(int), cudaMemcpyDeviceToHost, s));
  VBG_CUDA(cudaStreamSynchronize(s));
  *same = h == 0;
  return 0;
}

static int same_pattern_axpby(vbg_matrix* Y, double are, double aim, const vbg_matrix* X, double bre, double bim,
                              cudaStream_t s) {
  if (Y->nnz == 0) return 0;
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((Y->nnz + 255) / 256, sm_count() * 16));
  if (Y->dtype == VBG_C128)
    axpby_same_kernel<cplx><<<grid, 256, 0, s>>>(Y->nnz, are, aim, X->vals.as<cplx>(), bre, bim, Y->vals.as<cplx>());
  else
    axpby_same_kernel<double><<<grid, 256, 0, s>>>(Y->nnz, are, aim, X->vals.as<double>(), bre, bim,
                                                   Y->vals.as<double>());
  VBG_CUDA(cudaGetLastError());
  Y->invalidate_values();
  return 0;
}

// Fills a fresh matrix from an explicit pattern and per-slot source maps.
static int build_from_maps(const vbg_matrix* like, const std::vector<int>& rp, const std::vector<int>& ci,
                           const vbg_matrix* A, const std::vector<int>& mapA, double are, double aim,
                           const vbg_matrix* B, const std::vector<int>& mapB, double bre, double bim, int transpose,
                           vbg_matrix** out, cudaStream_t s) {
  auto d = std::make_unique<vbg_matrix>();
  d->dtype = like->dtype;
  d->device = like->device;
  int rc = build_structure(d.get(), like->n, like->h_bsz.data(), rp.data(), ci.data(), nullptr);
  if (rc) return rc;
  if ((rc = upload_structure(d.get(), s))) return rc;
  const size_t es = elem_size(d->dtype);
  if ((rc = d->vals.ensure(std::max<int64_t>(d->nnz, 1) * es))) return rc;
  if (d->nnzb > 0) {
    std::vector<int> out_row(d->nnzb);
    for (int i = 0; i < d->n; ++i)
      for (int p = d->h_row_ptr[i]; p < d->h_row_ptr[i + 1]; ++p) out_row[p] = i;
    DevBuf dmA, dmB, drow;
    if ((rc = drow.ensure(d->nnzb * sizeof(int)))) return rc;
    VBG_CUDA(cudaMemcpyAsync(drow.p, out_row.data(), d->nnzb * sizeof(int), cudaMemcpyHostToDevice, s));
    if (A) {
      if ((rc = dmA.ensure(d->nnzb * sizeof(int)))) return rc;
      VBG_CUDA(cudaMemcpyAsync(dmA.p, mapA.data(), d->nnzb * sizeof(int), cudaMemcpyHostToDevice, s));
    }
    if (B) {
      if ((rc = dmB.ensure(d->nnzb * sizeof(int)))) return rc;
      VBG_CUDA(cudaMemcpyAsync(dmB.p, mapB.data(), d->nnzb * sizeof(int), cudaMemcpyHostToDevice, s));
    }
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((d->nnzb + 7) / 8, sm_count() * 16));
    if (d->dtype == VBG_C128)
      gather_combine_kernel<cplx><<<grid, 256, 0, s>>>(
          d->nnzb, d->blk_off.as<int64_t>(), d->vals.as<cplx>(), drow.as<int>(), d->col_ind.as<int>(),
          d->bsz.as<int>(), A ? A->vals.as<cplx>() : nullptr, A ? A->blk_off.as<int64_t>() : nullptr,
          A ? dmA.as<int>() : nullptr, are, aim, B ? B->vals.as<cplx>() : nullptr,
          B ? B->blk_off.as<int64_t>() : nullptr, B ? dmB.as<int>() : nullptr, bre, bim, transpose);
    else
      gather_combine_kernel<double><<<grid, 256, 0, s>>>(
          d->nnzb, d->blk_off.as<int64_t>(), d->vals.as<double>(), drow.as<int>(), d->col_ind.as<int>(),
          d->bsz.as<int>(), A ? A->vals.as<double>() : nullptr, A ? A->blk_off.as<int64_t>() : nullptr,
          A ? dmA.as<int>() : nullptr, are, aim, B ? B->vals.as<double>() : nullptr,
          B ? B->blk_off.as<int64_t>() : nullptr, B ? dmB.as<int>() : nullptr, bre, bim, transpose);
    VBG_CUDA(cudaGetLastError());
    // the temporary maps are freed on return
    VBG_CUDA(cudaStreamSynchronize(s));
  }
  *out = d.release();
  return 0;
}

// Thread per block row: the merge of Y's and X's column lists of the row in
// the order of axpby.hpp's union fallback -- equal columns pair up one by
// one, so duplicate columns inside a row merge in order.  pass 0 counts the
// row's union slots into cnt[i]; pass 1 writes the union's columns and each
// slot's source slots in Y and X (-1: no block on that side).  A null Y
// pattern stands for an empty matrix (the result then has X's pattern).
__global__ void union_rows_kernel(int n, const int* __restrict__ yrp, const int* __restrict__ yci,
                                  const int* __restrict__ xrp, const int* __restrict__ xci, int pass,
                                  int* __restrict__ cnt, const int* __restrict__ urp, int* __restrict__ uci,
                                  int* __restrict__ uy, int* __restrict__ ux) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    int a = yrp ? yrp[i] : 0;
    const int ae = yrp ? yrp[i + 1] : 0;
    int b = xrp[i];
    const int be = xrp[i + 1];
    int o = pass ? urp[i] : 0;
    while (a < ae || b < be) {
      const int ja = a < ae ? yci[a] : INT32_MAX;
      const int jb = b < be ? xci[b] : INT32_MAX;
      const int j = min(ja, jb);
      if (pass) {
        uci[o] = j;
        uy[o] = ja == j ? a : -1;
        ux[o] = jb == j ? b : -1;
      }
      a += ja == j;
      b += jb == j;
      ++o;
    }
    if (!pass) cnt[i] = o;
  }
}

void move_into(vbg_matrix* dst, vbg_matrix* src);

// Y <- alpha X + beta Y on the union of the two patterns, or on X's pattern
// when Y's blocks do not contribute (ys == false).  Pattern and values are
// built on the device; the result replaces Y's contents.
static int axpby_union(vbg_matrix* Y, double are, double aim, const vbg_matrix* X, double bre, double bim, bool ys,
                       cudaStream_t s) {
  const int n = Y->n;
  int rc;
  DevBuf cnt(s), urp(s), uci(s), uy(s), ux(s);
  if ((rc = cnt.ensure((n + 1) * sizeof(int)))) return rc;
  if ((rc = urp.ensure((n + 1) * sizeof(int)))) return rc;
  VBG_CUDA(cudaMemsetAsync(cnt.p, 0, (n + 1) * sizeof(int), s));
  const int grid = std::max(1, std::min((n + 127) / 128, sm_count() * 8));
  const int* yrp = ys ? Y->row_ptr.as<int>() : nullptr;
  const int* yci = ys ? Y->col_ind.as<int>() : nullptr;
  if (n) {
    union_rows_kernel<<<grid, 128, 0, s>>>(n, yrp, yci, X->row_ptr.as<int>(), X->col_ind.as<int>(), 0, cnt.as<int>(),
                                          nullptr, nullptr, nullptr, nullptr);
    VBG_CUDA(cudaGetLastError());
  }
  if ((rc = exclusive_sum_int(cnt.as<int>(), urp.as<int>(), n + 1, s))) return rc;
  int total = 0;
  VBG_CUDA(cudaMemcpyAsync(&total, urp.as<int>() + n, sizeof(int), cudaMemcpyDeviceToHost, s));
  VBG_CUDA(cudaStreamSynchronize(s));
  if ((rc = uci.ensure(std::max(total, 1) * sizeof(int)))) return rc;
  if ((rc = uy.ensure(std::max(total, 1) * sizeof(int)))) return rc;
  if ((rc = ux.ensure(std::max(total, 1) * sizeof(int)))) return rc;
  if (n) {
    union_rows_kernel<<<grid, 128, 0, s>>>(n, yrp, yci, X->row_ptr.as<int>(), X->col_ind.as<int>(), 1, nullptr,
                                          urp.as<int>(), uci.as<int>(), uy.as<int>(), ux.as<int>());
    VBG_CUDA(cudaGetLastError());
  }
  auto d = std::make_unique<vbg_matrix>();
  d->dtype = Y->dtype;
  d->device = Y->device;
  if ((rc = adopt_device_structure(d.get(), Y, urp, uci, total, s))) return rc;
  const size_t es = elem_size(d->dtype);
  if ((rc = d->vals.ensure(std::max<int64_t>(d->nnz, 1) * es, s))) return rc;
  if (total) {
    const int g2 = std::max(1, std::min((total + 7) / 8, sm_count() * 16));
    if (d->dtype == VBG_C128)
      gather_combine_kernel<cplx><<<g2, 256, 0, s>>>(
          total, d->blk_off.as<int64_t>(), d->vals.as<cplx>(), nullptr, nullptr, d->bsz.as<int>(), X->vals.as<cplx>(),
          X->blk_off.as<int64_t>(), ux.as<int>(), are, aim, ys ? Y->vals.as<cplx>() : nullptr,
          Y->blk_off.as<int64_t>(), ys ? uy.as<int>() : nullptr, bre, bim, 0);
    else
      gather_combine_kernel<double><<<g2, 256, 0, s>>>(
          total, d->blk_off.as<int64_t>(), d->vals.as<double>(), nullptr, nullptr, d->bsz.as<int>(),
          X->vals.as<double>(), X->blk_off.as<int64_t>(), ux.as<int>(), are, aim,
          ys ? Y->vals.as<double>() : nullptr, Y->blk_off.as<int64_t>(), ys ? uy.as<int>() : nullptr, bre, bim, 0);
    VBG_CUDA(cudaGetLastError());
  }
  VBG_CUDA(cudaStreamSynchronize(s));
  move_into(Y, d.get());
  return 0;
}

// ------------------------------------------------------------ Hermitian completion
// Thread per block row i of C = U + strict_lower(U^H), U holding the upper
// block triangle: row i lists the mirrors of U's blocks (k, i), k < i (U's
// column view, rows ascending), then U's own blocks (i, j >= i); anything U
// holds below the diagonal is ignored (conjugate_transpose with mirror,
// ops/transpose.hpp:139-198).  pass 0 counts; pass 1 writes the columns, the
// source slot in U and whether the block is a mirror.
__global__ void herm_rows_kernel(int n, const int* __restrict__ urp, const int* __restrict__ uci,
                                 const int* __restrict__ cptr, const int* __restrict__ crow,
                                 const int* __restrict__ cslot, int pass, int* __restrict__ cnt,
                                 const int* __restrict__ rp, int* __restrict__ ci, int* __restrict__ src,
                                 unsigned char* __restrict__ tr) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    int o = pass ? rp[i] : 0;
    for (int p = cptr[i]; p < cptr[i + 1] && crow[p] < i; ++p) {
      if (pass) {
        ci[o] = crow[p];
        src[o] = cslot[p];
        tr[o] = 1;
      }
      ++o;
    }
    for (int q = urp[i]; q < urp[i + 1]; ++q)
      if (uci[q] >= i) {
        if (pass) {
          ci[o] = uci[q];
          src[o] = q;
          tr[o] = 0;
        }
        ++o;
      }
    if (!pass) cnt[i] = o;
  }
}

// Warp per block of C: a copy of U's block, or for a mirror the conjugate
// transpose of U's block (j, i): C(i, j)[q][t] = conj(U(j, i)[t][q]).
template <typename T>
__global__ void herm_gather_kernel(int64_t nout, const int64_t* __restrict__ out_off, const int* __restrict__ out_col,
                                   const int* __restrict__ bsz, T* __restrict__ out, const int* __restrict__ src,
                                   const unsigned char* __restrict__ tr, const int64_t* __restrict__ u_off,
                                   const T* __restrict__ U) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t p = blockIdx.x * (int64_t)(blockDim.x >> 5) + (threadIdx.x >> 5); p < nout; p += warps) {
    const int64_t o0 = out_off[p], len = out_off[p + 1] - o0;
    const int cj = bsz[out_col[p]];
    const int ri = (int)(len / cj);
    const T* sp = U + u_off[src[p]];
    const bool mirror = tr[p] != 0;
    for (int64_t e = lane; e < len; e += 32) {
      if (mirror) {
        const int64_t q = e / cj, t = e - q * cj;
        out[o0 + e] = conj_s(sp[t * ri + q]);
      } else {
        out[o0 + e] = sp[e];
      }
    }
  }
}

// (u + conj(l)) * 0.5, and the Hermitized diagonal element (its real part).
__device__ __forceinline__ double herm_avg(double u, double l) { return (u + l) * 0.5; }
__device__ __forceinline__ cplx herm_avg(cplx u, cplx l) { return {(u.re + l.re) * 0.5, (u.im - l.im) * 0.5}; }
__device__ __forceinline__ double herm_diag(double v) { return v; }
__device__ __forceinline__ cplx herm_diag(cplx v) { return {v.re, 0.0}; }

// Warp per block row: D <- (D + D^H) / 2 on its diagonal block
// (hermitize_diagonal_blocks, block_csr.hpp:1941-1966).  The lane of
// element (r, c), r < c, writes both (r, c) and (c, r).
template <typename T>
__global__ void hermitize_diag_kernel(int n, const int* __restrict__ diag, const int* __restrict__ bsz,
                                      const int64_t* __restrict__ off, T* __restrict__ vals) {
  const int lane = threadIdx.x & 31;
  const int warps = gridDim.x * (blockDim.x >> 5);
  for (int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); i < n; i += warps) {
    const int d = diag[i];
    if (d < 0) continue;
    const int r = bsz[i];
    T* D = vals + off[d];
    for (int e = lane; e < r * r; e += 32) {
      const int rr = e / r, cc = e - rr * r;
      if (rr == cc) {
        D[e] = herm_diag(D[e]);
      } else if (rr < cc) {
        const T avg = herm_avg(D[rr * r + cc], D[cc * r + rr]);
        D[rr * r + cc] = avg;
        D[cc * r + rr] = conj_s(avg);
      }
    }
  }
}

int complete_hermitian_dev(vbg_matrix* U, cudaStream_t s) {
  const int n = U->n;
  int rc;
  if ((rc = build_csc_dev(U, s))) return rc;
  DevBuf cnt(s), rp(s), ci(s), src(s), tr(s);
  if ((rc = cnt.ensure((n + 1) * sizeof(int)))) return rc;
  if ((rc = rp.ensure((n + 1) * sizeof(int)))) return rc;
  VBG_CUDA(cudaMemsetAsync(cnt.p, 0, (n + 1) * sizeof(int), s));
  const int grid = std::max(1, std::min((n + 127) / 128, sm_count() * 8));
  if (n) {
    herm_rows_kernel<<<grid, 128, 0, s>>>(n, U->row_ptr.as<int>(), U->col_ind.as<int>(), U->csc_ptr.as<int>(),
                                          U->csc_row.as<int>(), U->csc_slot.as<int>(), 0, cnt.as<int>(), nullptr,
                                          nullptr, nullptr, nullptr);
    VBG_CUDA(cudaGetLastError());
  }
  if ((rc = exclusive_sum_int(cnt.as<int>(), rp.as<int>(), n + 1, s))) return rc;
  int total = 0;
  VBG_CUDA(cudaMemcpyAsync(&total, rp.as<int>() + n, sizeof(int), cudaMemcpyDeviceToHost, s));
  VBG_CUDA(cudaStreamSynchronize(s));
  if ((rc = ci.ensure(std::max(total, 1) * sizeof(int)))) return rc;
  if ((rc = src.ensure(std::max(total, 1) * sizeof(int)))) return rc;
  if ((rc = tr.ensure(std::max(total, 1)))) return rc;
  if (n) {
    herm_rows_kernel<<<grid, 128, 0, s>>>(n, U->row_ptr.as<int>(), U->col_ind.as<int>(), U->csc_ptr.as<int>(),
                                          U->csc_row.as<int>(), U->csc_slot.as<int>(), 1, nullptr, rp.as<int>(),
                                          ci.as<int>(), src.as<int>(), tr.as<unsigned char>());
    VBG_CUDA(cudaGetLastError());
  }
  auto d = std::make_unique<vbg_matrix>();
  d->dtype = U->dtype;
  d->device = U->device;
  if ((rc = adopt_device_structure(d.get(), U, rp, ci, total, s))) return rc;
  const size_t es = elem_size(d->dtype);
  if ((rc = d->vals.ensure(std::max<int64_t>(d->nnz, 1) * es, s))) return rc;
  if (total) {
    const int g2 = std::max(1, std::min((total + 7) / 8, sm_count() * 16));
    const int g3 = std::max(1, std::min((n + 7) / 8, sm_count() * 16));
    if (d->dtype == VBG_C128) {
      herm_gather_kernel<cplx><<<g2, 256, 0, s>>>(total, d->blk_off.as<int64_t>(), d->col_ind.as<int>(),
                                                  d->bsz.as<int>(), d->vals.as<cplx>(), src.as<int>(),
                                                  tr.as<unsigned char>(), U->blk_off.as<int64_t>(), U->vals.as<cplx>());
      hermitize_diag_kernel<cplx><<<g3, 256, 0, s>>>(n, d->diag_slot.as<int>(), d->bsz.as<int>(),
                                                     d->blk_off.as<int64_t>(), d->vals.as<cplx>());
    } else {
      herm_gather_kernel<double><<<g2, 256, 0, s>>>(total, d->blk_off.as<int64_t>(), d->col_ind.as<int>(),
                                                    d->bsz.as<int>(), d->vals.as<double>(), src.as<int>(),
                                                    tr.as<unsigned char>(), U->blk_off.as<int64_t>(),
                                                    U->vals.as<double>());
      hermitize_diag_kernel<double><<<g3, 256, 0, s>>>(n, d->diag_slot.as<int>(), d->bsz.as<int>(),
                                                       d->blk_off.as<int64_t>(), d->vals.as<double>());
    }
    VBG_CUDA(cudaGetLastError());
  }
  VBG_CUDA(cudaStreamSynchronize(s));
  move_into(U, d.get());
  return 0;
}

// Moves the contents of `src` into `dst` (handle identity is kept).
void move_into(vbg_matrix* dst, vbg_matrix* src) {
  dst->graphs.clear();
  std::swap(dst->n, src->n);
  std::swap(dst->nnzb, src->nnzb);
  std::swap(dst->nnz, src->nnz);
  std::swap(dst->N, src->N);
  std::swap(dst->kind, src->kind);
  std::swap(dst->max_bs, src->max_bs);
  std::swap(dst->min_bs, src->min_bs);
  std::swap(dst->h_row_ptr, src->h_row_ptr);
  std::swap(dst->h_col_ind, src->h_col_ind);
  std::swap(dst->h_bsz, src->h_bsz);
  std::swap(dst->h_blk_off, src->h_blk_off);
  std::swap(dst->host_struct, src->host_struct);
  std::swap(dst->dup_cols, src->dup_cols);
  std::swap(dst->h_scal_off, src->h_scal_off);
  std::swap(dst->class_segs, src->class_segs);
  auto sw = [](DevBuf& a, DevBuf& b) { swap_mem(a, b); };
  sw(dst->row_ptr, src->row_ptr);
  sw(dst->col_ind, src->col_ind);
  sw(dst->bsz, src->bsz);
  sw(dst->scal_off, src->scal_off);
  sw(dst->blk_off, src->blk_off);
  sw(dst->diag_slot, src->diag_slot);
  sw(dst->row_perm, src->row_perm);
  sw(dst->slot_meta, src->slot_meta);
  sw(dst->vals, src->vals);
  dst->invalidate_structure();
}

__global__ void keep_kernel(const double* __restrict__ norms, int64_t n, double thr, unsigned char* keep) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    keep[i] = norms[i] >= thr ? 1 : 0;
}

int filter_blocks_impl(vbg_matrix* m, double thr, cudaStream_t s) {
  if (thr <= 0.0 || m->nnzb == 0) return 0;
  DevBuf norms(s), keep(s);
  int rc;
  if ((rc = norms.ensure(m->nnzb * sizeof(double)))) return rc;
  if ((rc = keep.ensure(m->nnzb))) return rc;
  if ((rc = block_norms_dev(m, norms.as<double>(), s))) return rc;
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((m->nnzb + 255) / 256, sm_count() * 16));
  keep_kernel<<<grid, 256, 0, s>>>(norms.as<double>(), m->nnzb, thr, keep.as<unsigned char>());
  VBG_CUDA(cudaGetLastError());
  return compact_by_mask_dev(m, keep.as<unsigned char>(), s);
}

}  // namespace vbg

using namespace vbg;

extern "C" {

int vbg_matrix_filter_blocks(vbg_matrix* m, double threshold, void* stream) {
  VBG_CHECK(m, VBG_E_ARG, "null matrix");
  return filter_blocks_impl(m, threshold, as_stream(stream));
}

int vbg_matrix_transpose(const vbg_matrix* m, vbg_matrix** out, void* stream) {
  VBG_CHECK(m && out, VBG_E_ARG, "null argument");
  cudaStream_t s = as_stream(stream);
  int rc0 = ensure_host_structure(m, s);
  if (rc0) return rc0;
  // rows of A^H = columns of A; within a row the source rows ascend
  std::vector<int> rp(m->n + 1, 0), ci(m->nnzb), map(m->nnzb);
  for (int64_t k = 0; k < m->nnzb; ++k) rp[m->h_col_ind[k] + 1]++;
  for (int j = 0; j < m->n; ++j) rp[j + 1] += rp[j];
  std::vector<int> fill(rp.begin(), rp.end() - 1);
  for (int i = 0; i < m->n; ++i)
    for (int k = m->h_row_ptr[i]; k < m->h_row_ptr[i + 1]; ++k) {
      const int p = fill[m->h_col_ind[k]]++;
      ci[p] = i;
      map[p] = k;
    }
  return build_from_maps(m, rp, ci, m, map, 1.0, 0.0, nullptr, {}, 0.0, 0.0, 1, out, s);
}

int vbg_matrix_axpby(vbg_matrix* Y, double are, double aim, const vbg_matrix* X, double bre, double bim,
                     void* stream) {
  VBG_CHECK(Y && X, VBG_E_ARG, "null matrix");
  VBG_CHECK(Y->dtype == X->dtype, VBG_E_ARG, "axpby: dtype mismatch");
  VBG_CHECK(Y->n == X->n && Y->h_bsz == X->h_bsz, VBG_E_ARG, "Matrix row count mismatch in axpby");
  cudaStream_t s = as_stream(stream);
  // axpby.hpp / block_csr.hpp:1250 fast paths: self-aliasing scales by
  // alpha + beta; alpha == 0 keeps Y's pattern; beta == 0 takes X's pattern.
  if (Y == X) return vbg_matrix_scale(Y, are + bre, aim + bim, stream);
  if (are == 0.0 && aim == 0.0) return vbg_matrix_scale(Y, bre, bim, stream);
  const bool beta_zero = bre == 0.0 && bim == 0.0;
  int rc = 0;
  bool same = false;
  if ((rc = same_pattern(Y, X, &same, s))) return rc;
  if (same) return same_pattern_axpby(Y, are, aim, X, bre, bim, s);
  // beta == 0 takes X's pattern; otherwise the union, columns ascending per
  // row (ops/axpby.hpp union fallback)
  const bool dup = Y->dup_cols || X->dup_cols;
  if ((rc = axpby_union(Y, are, aim, X, bre, bim, !beta_zero, s))) return rc;
  Y->dup_cols = beta_zero ? X->dup_cols : dup;
  return 0;
}

}  // extern "C"
