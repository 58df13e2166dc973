// Thresholded block SpGEMM  C = A B.
//
// Reference behaviour replaced (vbcsr/core/detail/ops/spmm/vbcsr.hpp:70-115
// VBCSRSpMMExecutor::run):
//   symbolic  ops/spmm/common.hpp:508-735: per C row, sum |A_ik|_F |B_kj|_F
//             per column j over the (A slot, B slot) pairs in slot order and
//             keep j iff the sum > threshold; columns sorted (:664, :668)
//   numeric   ops/spmm/vbcsr.hpp:206-471: per pair, skip when
//             |A_ik||B_kj| < threshold / max(1, nnzblk(A row i)) (:372, :386)
//             or when j is not in C's row; else C_ij += A_ik B_kj
//   filter    C.filter_blocks(threshold) (block_csr.hpp:1399-1528):
//             keep blocks with Frobenius norm >= threshold
//
// GPU layout: one warp per C row.  Symbolic: the warp walks the row's A
// slots in order; for each A slot the lanes take the B row's slots (distinct
// columns) and accumulate into an open-addressing table (shared memory, or a
// global-memory table for rows too wide for it), so every column's sum is
// formed in the reference's order with separately rounded products and adds
// -- the kept pattern is the reference's bit for bit.  Kept columns are
// compacted with warp ballots and bitonic-sorted.  Numeric: the warp maps
// C's columns in a table, then each lane multiplies one (A_ik, B_kj) block
// pair into its destination block; the Frobenius norms of the finished row
// are computed in the same kernel (the filter's keep flags), and the kept
// blocks are compacted afterwards.
#include <algorithm>
#include <cstring>
#include <numeric>
#include <vector>

#include <cub/device/device_scan.cuh>

#include "vbg_internal.cuh"

namespace vbg {

int block_norms_dev(const vbg_matrix* m, double* out, cudaStream_t s);
int compact_by_mask(vbg_matrix* m, const std::vector<unsigned char>& keep, cudaStream_t s);
int compact_by_mask_dev(vbg_matrix* m, const unsigned char* keep, cudaStream_t s);
int adopt_device_structure(vbg_matrix* m, const vbg_matrix* like, DevBuf& d_rp, DevBuf& d_ci, int64_t nnzb,
                           cudaStream_t s);

constexpr int kEmpty = -1;
constexpr int kSmemBudget = 96 * 1024;  // shared memory per CTA for the tables
constexpr int kMaxWarps = 8;

struct SymArgs {
  const int* a_rp;
  const int* a_ci;
  const double* nA;
  const int* b_rp;
  const int* b_ci;
  const double* nB;
  double thr;
  int serial_lanes;   // B has duplicate columns in a row: one lane at a time
  const int* rows;    // rows of this bin
  int nrows;
  int T;              // table entries (power of two)
  int pass;           // 0: count, 1: write sorted columns
  int* cnt;           // [n] kept columns per row (pass 0)
  const int* c_rp;    // pass 1
  int* c_ci;          // pass 1
  char* gtab;         // global tables (nullptr = shared memory)
  int* err;           // set on a table overflow (never expected)
};

__device__ __forceinline__ void bitonic_sort_warp(int* list, int L, int lane) {
  for (int k = 2; k <= L; k <<= 1) {
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int i = lane; i < L; i += 32) {
        const int ixj = i ^ j;
        if (ixj > i) {
          const int a = list[i], b = list[ixj];
          const bool up = (i & k) == 0;
          if ((a > b) == up) {
            list[i] = b;
            list[ixj] = a;
          }
        }
      }
      __syncwarp();
    }
  }
}

// Table layout per warp: keys int[T] | vals double[T] | list int[T/2]
__host__ __device__ inline size_t sym_table_bytes(int T) { return (size_t)T * 12 + (size_t)(T / 2) * 4 + 16; }

__global__ void spgemm_symbolic_kernel(SymArgs a) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  const int wpb = blockDim.x >> 5;
  const int T = a.T;
  const int mask = T - 1;
  const size_t tb = sym_table_bytes(T);
  const int gwarp = blockIdx.x * wpb + wib;
  unsigned char* base = a.gtab ? reinterpret_cast<unsigned char*>(a.gtab) + (size_t)gwarp * tb : smem + (size_t)wib * tb;
  double* vals = reinterpret_cast<double*>(base);
  int* keys = reinterpret_cast<int*>(base + (size_t)T * 8);
  int* list = keys + T;
  for (int w = gwarp; w < a.nrows; w += gridDim.x * wpb) {
    const int row = a.rows[w];
    for (int h = lane; h < T; h += 32) keys[h] = kEmpty;
    __syncwarp();
    for (int as = a.a_rp[row]; as < a.a_rp[row + 1]; ++as) {
      const int kk = a.a_ci[as];
      const double na = a.nA[as];
      const int b0 = a.b_rp[kk], b1 = a.b_rp[kk + 1];
      const int width = a.serial_lanes ? 1 : 32;
      for (int bc = b0; bc < b1; bc += width) {
        const int b = bc + lane;
        if (lane < width && b < b1) {
          const int j = a.b_ci[b];
          const double v = __dmul_rn(na, a.nB[b]);
          int h = j & mask;
          int probes = 0;
          while (true) {
            int k = keys[h];
            if (k == kEmpty) {
              k = atomicCAS(&keys[h], kEmpty, j);
              if (k == kEmpty) {
                vals[h] = v;
                break;
              }
            }
            if (k == j) {
              vals[h] = __dadd_rn(vals[h], v);
              break;
            }
            h = (h + 1) & mask;
            if (++probes > T) {
              atomicExch(a.err, 1);
              break;
            }
          }
        }
        if (a.serial_lanes) __syncwarp();
      }
      __syncwarp();
    }
    // kept columns: sum > threshold (common.hpp:664)
    int base_pos = 0;
    for (int h0 = 0; h0 < T; h0 += 32) {
      const int h = h0 + lane;
      const bool kept = keys[h] != kEmpty && vals[h] > a.thr;
      const unsigned bal = __ballot_sync(0xffffffffu, kept);
      if (a.pass == 1 && kept) list[base_pos + __popc(bal & ((1u << lane) - 1u))] = keys[h];
      base_pos += __popc(bal);
    }
    if (a.pass == 0) {
      if (lane == 0) a.cnt[row] = base_pos;
    } else if (base_pos > 0) {
      int L = 1;
      while (L < base_pos) L <<= 1;
      for (int i = base_pos + lane; i < L; i += 32) list[i] = 0x7fffffff;
      __syncwarp();
      bitonic_sort_warp(list, L, lane);
      int* out = a.c_ci + a.c_rp[row];
      for (int i = lane; i < base_pos; i += 32) out[i] = list[i];
    }
    __syncwarp();
  }
}

struct NumArgs {
  const int* a_rp;
  const int* a_ci;
  const int64_t* a_off;
  const double* nA;
  const int* b_rp;
  const int* b_ci;
  const int64_t* b_off;
  const double* nB;
  const int* bsz;
  const int* c_rp;
  const int* c_ci;
  const int64_t* c_off;
  double thr;
  int serial_lanes;
  const int* rows;
  int nrows;
  int T;
  char* gtab;
  unsigned char* keep;  // per C slot
  unsigned long long* products;
  int* err;
};

// C(r x c) += A(r x inner) B(inner x c), one lane.
template <typename T, int CC>
__device__ __forceinline__ void block_gemm_fixed(const T* __restrict__ ap, const T* __restrict__ bp, T* cp, int r,
                                                 int inner) {
  for (int t = 0; t < r; ++t) {
    T acc[CC];
#pragma unroll
    for (int u = 0; u < CC; ++u) acc[u] = cp[t * CC + u];
    for (int q = 0; q < inner; ++q) {
      const T x = ap[t * inner + q];
#pragma unroll
      for (int u = 0; u < CC; ++u) acc[u] = fma_s(x, bp[q * CC + u], acc[u]);
    }
#pragma unroll
    for (int u = 0; u < CC; ++u) cp[t * CC + u] = acc[u];
  }
}

template <typename T>
__device__ void block_gemm(const T* __restrict__ ap, const T* __restrict__ bp, T* cp, int r, int inner, int c) {
  switch (c) {
    case 1: block_gemm_fixed<T, 1>(ap, bp, cp, r, inner); return;
    case 2: block_gemm_fixed<T, 2>(ap, bp, cp, r, inner); return;
    case 3: block_gemm_fixed<T, 3>(ap, bp, cp, r, inner); return;
    case 4: block_gemm_fixed<T, 4>(ap, bp, cp, r, inner); return;
    case 5: block_gemm_fixed<T, 5>(ap, bp, cp, r, inner); return;
    case 6: block_gemm_fixed<T, 6>(ap, bp, cp, r, inner); return;
    case 7: block_gemm_fixed<T, 7>(ap, bp, cp, r, inner); return;
    case 8: block_gemm_fixed<T, 8>(ap, bp, cp, r, inner); return;
    default:
      for (int t = 0; t < r; ++t)
        for (int q = 0; q < inner; ++q) {
          const T x = ap[t * inner + q];
          for (int u = 0; u < c; ++u) cp[t * c + u] = fma_s(x, bp[q * c + u], cp[t * c + u]);
        }
  }
}

__device__ __forceinline__ double sq_mag(double v) { return __dmul_rn(v, v); }
__device__ __forceinline__ double sq_mag(cplx v) { return fma(v.re, v.re, __dmul_rn(v.im, v.im)); }

// Table layout per warp: keys int[T] | dest int[T]
__host__ __device__ inline size_t num_table_bytes(int T) { return (size_t)T * 8 + 16; }

template <typename T>
__global__ void spgemm_numeric_kernel(NumArgs a, const T* __restrict__ A, const T* __restrict__ B, T* C) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  const int wpb = blockDim.x >> 5;
  const int TT = a.T;
  const int mask = TT - 1;
  const size_t tb = num_table_bytes(TT);
  const int gwarp = blockIdx.x * wpb + wib;
  unsigned char* base = a.gtab ? reinterpret_cast<unsigned char*>(a.gtab) + (size_t)gwarp * tb : smem + (size_t)wib * tb;
  int* keys = reinterpret_cast<int*>(base);
  int* dest = keys + TT;
  unsigned long long prods = 0;
  for (int w = gwarp; w < a.nrows; w += gridDim.x * wpb) {
    const int row = a.rows[w];
    const int c0 = a.c_rp[row], c1 = a.c_rp[row + 1];
    for (int h = lane; h < TT; h += 32) keys[h] = kEmpty;
    __syncwarp();
    // map C's columns -> slots (distinct, sorted)
    for (int p = c0 + lane; p < c1; p += 32) {
      const int j = a.c_ci[p];
      int h = j & mask;
      int probes = 0;
      while (atomicCAS(&keys[h], kEmpty, j) != kEmpty) {
        h = (h + 1) & mask;
        if (++probes > TT) {
          atomicExch(a.err, 2);
          break;
        }
      }
      dest[h] = p;
    }
    __syncwarp();
    const int r = a.bsz[row];
    const int row_count = a.a_rp[row + 1] - a.a_rp[row];
    const double row_eps = a.thr / (double)max(1, row_count);
    for (int as = a.a_rp[row]; as < a.a_rp[row + 1]; ++as) {
      const int kk = a.a_ci[as];
      const int inner = a.bsz[kk];
      const double na = a.nA[as];
      const T* ap = A + a.a_off[as];
      const int b0 = a.b_rp[kk], b1 = a.b_rp[kk + 1];
      const int width = a.serial_lanes ? 1 : 32;
      for (int bc = b0; bc < b1; bc += width) {
        const int b = bc + lane;
        if (lane < width && b < b1 && !(na * a.nB[b] < row_eps)) {
          const int j = a.b_ci[b];
          int h = j & mask;
          int d = -1;
          for (int probes = 0; probes <= TT; ++probes) {
            const int k = keys[h];
            if (k == j) {
              d = dest[h];
              break;
            }
            if (k == kEmpty) break;
            h = (h + 1) & mask;
          }
          if (d >= 0) {
            block_gemm<T>(ap, B + a.b_off[b], C + a.c_off[d], r, inner, a.bsz[j]);
            ++prods;
          }
        }
        if (a.serial_lanes) __syncwarp();
      }
      __syncwarp();
    }
    // fused filter: Frobenius norm of each finished block of the row
    for (int p = c0 + lane; p < c1; p += 32) {
      double sum = 0.0;
      for (int64_t e = a.c_off[p]; e < a.c_off[p + 1]; ++e) sum = __dadd_rn(sum, sq_mag(C[e]));
      a.keep[p] = (a.thr <= 0.0 || sqrt(sum) >= a.thr) ? 1 : 0;
    }
    __syncwarp();
  }
  if (prods) atomicAdd(a.products, prods);
}

static int next_pow2(int64_t v) {
  int p = 32;
  while (p < v) p <<= 1;
  return p;
}

struct Bin {
  int T;
  std::vector<int> rows;
};

// Groups rows by table size.
static std::vector<Bin> make_bins(const std::vector<int64_t>& need) {
  std::map<int, std::vector<int>> by;
  for (size_t i = 0; i < need.size(); ++i)
    if (need[i] >= 0) by[next_pow2(need[i])].push_back((int)i);
  std::vector<Bin> out;
  for (auto& kv : by) out.push_back({kv.first, std::move(kv.second)});
  return out;
}

static bool has_duplicate_columns(const vbg_matrix* m) {
  for (int i = 0; i < m->n; ++i)
    for (int p = m->h_row_ptr[i] + 1; p < m->h_row_ptr[i + 1]; ++p)
      if (m->h_col_ind[p] == m->h_col_ind[p - 1]) return true;
  return false;
}

template <typename F>
static int launch_binned(const std::vector<Bin>& bins, size_t (*table_bytes)(int), DevBuf& rows_dev, DevBuf& gtab,
                         cudaStream_t s, F&& launch) {
  size_t total_rows = 0;
  for (auto& b : bins) total_rows += b.rows.size();
  std::vector<int> all;
  all.reserve(total_rows);
  for (auto& b : bins) all.insert(all.end(), b.rows.begin(), b.rows.end());
  int rc = rows_dev.ensure(std::max<size_t>(all.size(), 1) * sizeof(int));
  if (rc) return rc;
  if (!all.empty()) VBG_CUDA(cudaMemcpyAsync(rows_dev.p, all.data(), all.size() * sizeof(int), cudaMemcpyHostToDevice, s));
  size_t off = 0;
  for (auto& b : bins) {
    const size_t tb = table_bytes(b.T);
    const int nrows = (int)b.rows.size();
    const int* rows = rows_dev.as<int>() + off;
    off += b.rows.size();
    if (tb <= (size_t)kSmemBudget) {
      const int wpb = (int)std::max<size_t>(1, std::min<size_t>(kMaxWarps, kSmemBudget / tb));
      const int grid = std::max(1, std::min((nrows + wpb - 1) / wpb, sm_count() * 8));
      if ((rc = launch(rows, nrows, b.T, grid, wpb, (size_t)wpb * tb, (char*)nullptr))) return rc;
    } else {
      const int wpb = 4;
      const int grid = std::max(1, std::min((nrows + wpb - 1) / wpb, sm_count() * 2));
      if ((rc = gtab.ensure((size_t)grid * wpb * tb))) return rc;
      if ((rc = launch(rows, nrows, b.T, grid, wpb, (size_t)0, gtab.as<char>()))) return rc;
    }
  }
  return 0;
}

static size_t sym_tb(int T) { return sym_table_bytes(T); }
static size_t num_tb(int T) { return num_table_bytes(T); }

}  // namespace vbg

using namespace vbg;

extern "C" int vbg_spgemm(const vbg_matrix* A, const vbg_matrix* B, double thr, vbg_matrix** Cout, int64_t* stats,
                          void* stream) {
  VBG_CHECK(A && B && Cout, VBG_E_ARG, "null argument");
  VBG_CHECK(A->dtype == B->dtype, VBG_E_ARG, "A and B must have the same dtype");
  VBG_CHECK(A->n == B->n && A->h_bsz == B->h_bsz, VBG_E_ARG, "spmm: A's columns and B's rows differ");
  cudaStream_t s = as_stream(stream);
  const int n = A->n;
  int rc;
  // block norms of both operands (cached per call)
  DevBuf nA, nB, cnt, err, gtab, rows_dev;
  if ((rc = nA.ensure(std::max<int64_t>(A->nnzb, 1) * 8))) return rc;
  if ((rc = nB.ensure(std::max<int64_t>(B->nnzb, 1) * 8))) return rc;
  if ((rc = block_norms_dev(A, nA.as<double>(), s))) return rc;
  if ((rc = block_norms_dev(B, nB.as<double>(), s))) return rc;
  if ((rc = cnt.ensure((n + 1) * sizeof(int)))) return rc;
  if ((rc = err.ensure(16))) return rc;
  VBG_CUDA(cudaMemsetAsync(err.p, 0, 16, s));
  VBG_CUDA(cudaMemsetAsync(cnt.p, 0, (n + 1) * sizeof(int), s));
  const int serial_b = has_duplicate_columns(B) ? 1 : 0;

  // symbolic table sizes: 2 * min(sum of B row lengths, n) + 1 (common.hpp:600-616)
  std::vector<int64_t> need(n, -1);
  for (int i = 0; i < n; ++i) {
    int64_t bound = 0;
    for (int p = A->h_row_ptr[i]; p < A->h_row_ptr[i + 1]; ++p) {
      const int k = A->h_col_ind[p];
      bound += B->h_row_ptr[k + 1] - B->h_row_ptr[k];
    }
    if (bound == 0) continue;
    bound = std::min<int64_t>(bound, n);
    need[i] = 2 * bound + 1;
  }
  auto sym_bins = make_bins(need);
  SymArgs sa{};
  sa.a_rp = A->row_ptr.as<int>();
  sa.a_ci = A->col_ind.as<int>();
  sa.nA = nA.as<double>();
  sa.b_rp = B->row_ptr.as<int>();
  sa.b_ci = B->col_ind.as<int>();
  sa.nB = nB.as<double>();
  sa.thr = thr;
  sa.serial_lanes = serial_b;
  sa.cnt = cnt.as<int>();
  sa.err = err.as<int>();
  auto sym_launch = [&](int pass, const int* c_rp, int* c_ci) {
    return launch_binned(sym_bins, sym_tb, rows_dev, gtab, s,
                         [&](const int* rows, int nrows, int T, int grid, int wpb, size_t smem, char* gt) -> int {
                           SymArgs x = sa;
                           x.rows = rows;
                           x.nrows = nrows;
                           x.T = T;
                           x.pass = pass;
                           x.c_rp = c_rp;
                           x.c_ci = c_ci;
                           x.gtab = gt;
                           if (smem > 48 * 1024)
                             VBG_CUDA(cudaFuncSetAttribute(spgemm_symbolic_kernel,
                                                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
                           spgemm_symbolic_kernel<<<grid, wpb * 32, smem, s>>>(x);
                           VBG_CUDA(cudaGetLastError());
                           return 0;
                         });
  };
  if ((rc = sym_launch(0, nullptr, nullptr))) return rc;
  // C's row pointers: exclusive scan of the per-row counts on the device
  DevBuf d_crp, d_cci, scan_tmp;
  if ((rc = d_crp.ensure((n + 1) * sizeof(int)))) return rc;
  size_t scan_bytes = 0;
  VBG_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, cnt.as<int>(), d_crp.as<int>(), n + 1, s));
  if ((rc = scan_tmp.ensure(std::max<size_t>(scan_bytes, 16)))) return rc;
  VBG_CUDA(cub::DeviceScan::ExclusiveSum(scan_tmp.p, scan_bytes, cnt.as<int>(), d_crp.as<int>(), n + 1, s));
  int cnnzb_i = 0;
  VBG_CUDA(cudaMemcpyAsync(&cnnzb_i, d_crp.as<int>() + n, sizeof(int), cudaMemcpyDeviceToHost, s));
  VBG_CUDA(cudaStreamSynchronize(s));
  const int64_t cnnzb = cnnzb_i;
  if ((rc = d_cci.ensure(std::max<int64_t>(cnnzb, 1) * sizeof(int)))) return rc;
  if ((rc = sym_launch(1, d_crp.as<int>(), d_cci.as<int>()))) return rc;
  int herr[4] = {0, 0, 0, 0};
  VBG_CUDA(cudaMemcpyAsync(herr, err.p, 16, cudaMemcpyDeviceToHost, s));
  VBG_CUDA(cudaStreamSynchronize(s));
  VBG_CHECK(herr[0] == 0, VBG_E_DEVICE, "Hash table full in symbolic phase");

  // result matrix on the symbolic pattern (rows sorted by the symbolic
  // kernel); its structure metadata is built on the device
  auto C = std::make_unique<vbg_matrix>();
  C->dtype = A->dtype;
  C->device = A->device;
  if ((rc = adopt_device_structure(C.get(), A, d_crp, d_cci, cnnzb, s))) return rc;
  const std::vector<int>& crp = C->h_row_ptr;
  const size_t es = elem_size(C->dtype);
  if ((rc = C->vals.ensure(std::max<int64_t>(C->nnz, 1) * es))) return rc;
  VBG_CUDA(cudaMemsetAsync(C->vals.p, 0, std::max<int64_t>(C->nnz, 1) * es, s));
  DevBuf keep, prods;
  if ((rc = keep.ensure(std::max<int64_t>(cnnzb, 1)))) return rc;
  if ((rc = prods.ensure(16))) return rc;
  VBG_CUDA(cudaMemsetAsync(prods.p, 0, 16, s));

  std::vector<int64_t> cneed(n, -1);
  for (int i = 0; i < n; ++i)
    if (crp[i + 1] > crp[i]) cneed[i] = 2 * (int64_t)(crp[i + 1] - crp[i]) + 1;
  auto num_bins = make_bins(cneed);
  NumArgs na{};
  na.a_rp = A->row_ptr.as<int>();
  na.a_ci = A->col_ind.as<int>();
  na.a_off = A->blk_off.as<int64_t>();
  na.nA = nA.as<double>();
  na.b_rp = B->row_ptr.as<int>();
  na.b_ci = B->col_ind.as<int>();
  na.b_off = B->blk_off.as<int64_t>();
  na.nB = nB.as<double>();
  na.bsz = A->bsz.as<int>();
  na.c_rp = C->row_ptr.as<int>();
  na.c_ci = C->col_ind.as<int>();
  na.c_off = C->blk_off.as<int64_t>();
  na.thr = thr;
  na.serial_lanes = serial_b;
  na.keep = keep.as<unsigned char>();
  na.products = prods.as<unsigned long long>();
  na.err = err.as<int>();
  rc = launch_binned(num_bins, num_tb, rows_dev, gtab, s,
                     [&](const int* rows, int nrows, int T, int grid, int wpb, size_t smem, char* gt) -> int {
                       NumArgs x = na;
                       x.rows = rows;
                       x.nrows = nrows;
                       x.T = T;
                       x.gtab = gt;
                       if (C->dtype == VBG_C128) {
                         if (smem > 48 * 1024)
                           VBG_CUDA(cudaFuncSetAttribute(spgemm_numeric_kernel<cplx>,
                                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
                         spgemm_numeric_kernel<cplx><<<grid, wpb * 32, smem, s>>>(x, A->vals.as<cplx>(),
                                                                                  B->vals.as<cplx>(), C->vals.as<cplx>());
                       } else {
                         if (smem > 48 * 1024)
                           VBG_CUDA(cudaFuncSetAttribute(spgemm_numeric_kernel<double>,
                                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
                         spgemm_numeric_kernel<double><<<grid, wpb * 32, smem, s>>>(
                             x, A->vals.as<double>(), B->vals.as<double>(), C->vals.as<double>());
                       }
                       VBG_CUDA(cudaGetLastError());
                       return 0;
                     });
  if (rc) return rc;
  unsigned long long hprods = 0;
  VBG_CUDA(cudaMemcpyAsync(&hprods, prods.p, 8, cudaMemcpyDeviceToHost, s));
  VBG_CUDA(cudaMemcpyAsync(herr, err.p, 16, cudaMemcpyDeviceToHost, s));
  VBG_CUDA(cudaStreamSynchronize(s));
  VBG_CHECK(herr[0] == 0, VBG_E_DEVICE, "Hash table full during SpGEMM numeric phase");
  const int64_t sym_blocks = cnnzb;
  if (thr > 0.0 && (rc = compact_by_mask_dev(C.get(), keep.as<unsigned char>(), s))) return rc;
  if (stats) {
    stats[0] = sym_blocks;
    stats[1] = C->nnzb;
    stats[2] = (int64_t)hprods;
    stats[3] = -1;
  }
  *Cout = C.release();
  return 0;
}
