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

constexpr int kEmpty = -1;
constexpr int kSmemBudget = 96 * 1024;  // shared memory per CTA for the tables
constexpr int kMaxWarps = 8;
constexpr int64_t kNumRowSmem = 96 * 1024;  // largest row region kept in shared memory
constexpr int kNumWarps = 4;                // warps of a numeric CTA (one C row)

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
  int region;           // bytes of one CTA's row region (table + accumulators,
                        // or the table alone in global scratch)
  char* gtab;           // global regions (rows too wide for shared memory)
  unsigned char* keep;  // per C slot
  unsigned long long* products;
  int* err;
};

__device__ __forceinline__ double sq_mag(double v) { return __dmul_rn(v, v); }
__device__ __forceinline__ double sq_mag(cplx v) { return fma(v.re, v.re, __dmul_rn(v.im, v.im)); }

// Column table of one C row: TT entries (a power of two >= 2 cnt + 1, at
// least 32) of keys (block column) and row-local slots; the row's
// accumulators follow at a 16-byte boundary.
__host__ __device__ inline int num_table_size(int cnt) {
  int t = 32;
  while (t < 2 * cnt + 1) t <<= 1;
  return t;
}
__host__ __device__ inline size_t num_acc_offset(int TT) { return ((size_t)TT * 8 + 15) / 16 * 16; }

// Per-warp shared memory of the numeric kernel: the staged A block (8 rows of
// kAsStride scalars; the odd stride keeps the rows in distinct banks), then
// the pair list of one batch: first output, columns, accumulator offset and
// B offset of each pair.
constexpr int kAsStride = 9;
template <typename T>
__host__ __device__ constexpr int num_stage_bytes() {
  return (8 * kAsStride * (int)sizeof(T) + 15) / 16 * 16;
}
template <typename T>
__host__ __device__ constexpr int num_warp_bytes() {
  return num_stage_bytes<T>() + 32 * (3 * 4 + 8);
}

// floor(e / c) for 0 <= e < 64, 1 <= c <= 8 as (e * ceil(2^16 / c)) >> 16:
// the rounding error of the reciprocal stays below 64 / 2^16, less than the
// distance 1/8 from e / c to the next integer.
__constant__ int c_recip16[9] = {0, 65536, 32768, 21846, 16384, 13108, 10923, 9363, 8192};

// Real blocks of at most 8 x 8 use the FP64 tensor-core MMA.
template <typename T, int R>
constexpr bool kDmma = sizeof(T) == sizeof(double) && R != 0;

// D = A B + C for one 8 x 8 x 4 FP64 tile (mma.sync m8n8k4, row.col): lane l
// holds A(l / 4, l % 4), B(l % 4, l / 4) and C(l / 4, 2 (l % 4) + {0, 1}).
__device__ __forceinline__ void dmma_884(double& c0, double& c1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}

// The listed pairs of one batch on the tensor cores, one pair per step: the
// B block (inner x c, zero-padded to 8 x 8) and the C block's accumulators
// (r x c) as fragments, one MMA per four of the inner index.  The next
// pair's fragments are loaded before this pair's MMA (the pairs of a batch
// write distinct C blocks).
template <int R>
__device__ __forceinline__ void num_pairs_dmma(const int* Lc, const int* Ld, const int64_t* Lb, int np, int inner,
                                               double a0f, double a1f, const double* __restrict__ B, double* acc,
                                               int lane) {
  const int gq = lane >> 2, t4 = lane & 3;
  double b0, b1, c0, c1;
  int cc;
  double* cp;
  auto load = [&](int p) {
    cc = Lc[p];
    const double* bp = B + Lb[p];
    b0 = (t4 < inner && gq < cc) ? bp[t4 * cc + gq] : 0.0;
    b1 = (t4 + 4 < inner && gq < cc) ? bp[(t4 + 4) * cc + gq] : 0.0;
    cp = acc + Ld[p] + gq * cc + 2 * t4;
    c0 = (gq < R && 2 * t4 < cc) ? cp[0] : 0.0;
    c1 = (gq < R && 2 * t4 + 1 < cc) ? cp[1] : 0.0;
  };
  load(0);
  for (int p = 0; p < np; ++p) {
    const double pb0 = b0, pb1 = b1;
    double pc0 = c0, pc1 = c1;
    const int pcc = cc;
    double* pcp = cp;
    if (p + 1 < np) load(p + 1);
    dmma_884(pc0, pc1, a0f, pb0);
    if (inner > 4) dmma_884(pc0, pc1, a1f, pb1);
    if (gq < R && 2 * t4 < pcc) pcp[0] = pc0;
    if (gq < R && 2 * t4 + 1 < pcc) pcp[1] = pc1;
  }
}

// The products of one C row done by one warp of the row's CTA (block rows R;
// R = 0: any size, A read from global memory).  For each A slot (i, k) in
// order the warp stages A_ik, and its lanes take 32 slots (k, j) of B's row
// k at a time: a pair is skipped when |A_ik| |B_kj| < threshold /
// max(1, nnzb(A row i)) or when j is not in C's row, and kept only when C's
// row-local slot d of j belongs to this warp (d mod warps == warp), so every
// C element is updated by one warp in the reference's pair order.  The kept
// pairs of the batch are listed with their first output index (prefix sum of
// r x c) and their outputs are spread over the lanes: lane g computes C_ij(t,
// u) += sum_q A_ik(t, q) B_kj(q, u) as one fused multiply-add chain from the
// current value, consecutive lanes on consecutive u of one block, so the B
// block and the accumulators are read in contiguous runs.  The pairs of one
// batch write distinct C blocks (B's row has distinct columns; else the
// batch is one pair).
template <typename T, int R>
__device__ __forceinline__ void num_row(const NumArgs& a, const T* __restrict__ A, const T* __restrict__ B, T* acc,
                                        const int* keys, const int* slot, int TT, int row, int c0, int64_t rbase,
                                        unsigned char* wsm, int lane, int wib, int W, unsigned long long& prods) {
  T* As = reinterpret_cast<T*>(wsm);
  int* Ls = reinterpret_cast<int*>(wsm + num_stage_bytes<T>());
  int* Lc = Ls + 32;
  int* Ld = Lc + 32;
  int64_t* Lb = reinterpret_cast<int64_t*>(Ld + 32);
  const int mask = TT - 1;
  const int a0 = a.a_rp[row], a1 = a.a_rp[row + 1];
  const double row_eps = a.thr / (double)max(1, a1 - a0);
  const int width = a.serial_lanes ? 1 : 32;
  const int r = R ? R : a.bsz[row];
  for (int as = a0; as < a1; ++as) {
    const int kk = a.a_ci[as];
    const int inner = a.bsz[kk];
    const double na = a.nA[as];
    const T* ap = A + a.a_off[as];
    double a0f = 0.0, a1f = 0.0;  // A_ik as the two k-halves of an m8n8k4 A fragment
    if constexpr (kDmma<T, R>) {
      const int gq = lane >> 2, t4 = lane & 3;
      if (gq < R && t4 < inner) a0f = reinterpret_cast<const double*>(ap)[gq * inner + t4];
      if (gq < R && t4 + 4 < inner) a1f = reinterpret_cast<const double*>(ap)[gq * inner + t4 + 4];
    } else if constexpr (R != 0) {
      __syncwarp();
      for (int e = lane; e < R * inner; e += 32) {
        const int t = e / inner;
        As[t * kAsStride + (e - t * inner)] = ap[e];
      }
      __syncwarp();
    }
    const int b0 = a.b_rp[kk], b1 = a.b_rp[kk + 1];
    for (int bc = b0; bc < b1; bc += width) {
      const int b = bc + lane;
      int d = -1, j = 0;
      if (lane < width && b < b1 && !(na * a.nB[b] < row_eps)) {
        j = a.b_ci[b];
        int h = j & mask;
        for (int probes = 0; probes <= TT; ++probes) {
          const int key = keys[h];
          if (key == j) {
            d = slot[h];
            break;
          }
          if (key == kEmpty) break;
          h = (h + 1) & mask;
        }
        if (d >= 0 && d % W != wib) d = -1;
      }
      const unsigned m = __ballot_sync(0xffffffffu, d >= 0);
      if (m == 0) continue;
      const int c = d >= 0 ? a.bsz[j] : 0;
      const int nout = r * c;
      int incl = nout, total = 0;
      if constexpr (!kDmma<T, R>) {
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
          const int y = __shfl_up_sync(0xffffffffu, incl, off);
          if (lane >= off) incl += y;
        }
        total = __shfl_sync(0xffffffffu, incl, 31);
      }
      if (d >= 0) {
        const int pos = __popc(m & ((1u << lane) - 1u));
        Ls[pos] = incl - nout;
        Lc[pos] = c;
        Ld[pos] = (int)(a.c_off[c0 + d] - rbase);
        Lb[pos] = a.b_off[b];
      }
      const int np = __popc(m);
      __syncwarp();
      if constexpr (kDmma<T, R>) {
        num_pairs_dmma<R>(Lc, Ld, Lb, np, inner, a0f, a1f, reinterpret_cast<const double*>(B),
                          reinterpret_cast<double*>(acc), lane);
        __syncwarp();
        if (lane == 0) prods += np;
        continue;
      }
      for (int g = lane; g < total; g += 32) {
        int lo = 0, hi = np - 1;
        while (lo < hi) {
          const int mid = (lo + hi + 1) >> 1;
          if (Ls[mid] <= g) lo = mid;
          else hi = mid - 1;
        }
        const int e = g - Ls[lo], cc = Lc[lo];
        const int t = R ? (e * c_recip16[cc]) >> 16 : e / cc;
        const int u = e - t * cc;
        T* cp = acc + Ld[lo] + e;
        const T* bp = B + Lb[lo] + u;
        T v = *cp;
        if constexpr (R != 0) {
#pragma unroll
          for (int q = 0; q < 8; ++q)
            if (q < inner) v = fma_s(As[t * kAsStride + q], bp[q * cc], v);
        } else {
          for (int q = 0; q < inner; ++q) v = fma_s(ap[t * inner + q], bp[q * cc], v);
        }
        *cp = v;
      }
      __syncwarp();
      if (lane == 0) prods += np;
    }
  }
}

// One CTA per C row of the bin (block rows R for all of them; R = 0: any
// size; one kernel per row size keeps each one's register allocation its
// own).  The row's column table and accumulators live in the CTA's shared
// memory, or -- for rows too wide for it -- the table in global scratch and
// the accumulators in the row's own slice of C (zeroed first).  Afterwards
// the Frobenius norm of every finished block gives the filter's keep flag,
// and a shared-memory row is written out.
template <typename T, int R>
__global__ void __launch_bounds__(128) spgemm_numeric_kernel(NumArgs a, const T* __restrict__ A,
                                                             const T* __restrict__ B, T* C) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  const int W = blockDim.x >> 5;
  unsigned char* wsm = smem + (size_t)wib * num_warp_bytes<T>();
  unsigned char* region = a.gtab ? reinterpret_cast<unsigned char*>(a.gtab) + (size_t)blockIdx.x * a.region
                                 : smem + (size_t)W * num_warp_bytes<T>();
  unsigned long long prods = 0;
  for (int w = blockIdx.x; w < a.nrows; w += gridDim.x) {
    const int row = a.rows[w];
    const int c0 = a.c_rp[row], c1 = a.c_rp[row + 1];
    const int TT = num_table_size(c1 - c0);
    int* keys = reinterpret_cast<int*>(region);
    int* slot = keys + TT;
    const int64_t rbase = a.c_off[c0], E = a.c_off[c1] - rbase;
    T* acc = a.gtab ? C + rbase : reinterpret_cast<T*>(region + num_acc_offset(TT));
    for (int h = threadIdx.x; h < TT; h += blockDim.x) keys[h] = kEmpty;
    for (int64_t e = threadIdx.x; e < E; e += blockDim.x) acc[e] = zero_s<T>();
    __syncthreads();
    for (int p = c0 + threadIdx.x; p < c1; p += blockDim.x) {
      const int j = a.c_ci[p];
      int h = j & (TT - 1);
      int probes = 0;
      while (atomicCAS(&keys[h], kEmpty, j) != kEmpty) {
        h = (h + 1) & (TT - 1);
        if (++probes > TT) {
          atomicExch(a.err, 2);
          break;
        }
      }
      slot[h] = p - c0;
    }
    __syncthreads();
    num_row<T, R>(a, A, B, acc, keys, slot, TT, row, c0, rbase, wsm, lane, wib, W, prods);
    __syncthreads();
    // fused filter: Frobenius norm of each finished block of the row
    for (int p = c0 + threadIdx.x; p < c1; p += blockDim.x) {
      double sum = 0.0;
      for (int64_t e = a.c_off[p] - rbase; e < a.c_off[p + 1] - rbase; ++e) sum = __dadd_rn(sum, sq_mag(acc[e]));
      a.keep[p] = (a.thr <= 0.0 || sqrt(sum) >= a.thr) ? 1 : 0;
    }
    if (!a.gtab)
      for (int64_t e = threadIdx.x; e < E; e += blockDim.x) C[rbase + e] = acc[e];
    __syncthreads();
  }
  if (prods) atomicAdd(a.products, prods);
}

template <typename T, int R>
static int launch_numeric_r(const NumArgs& x, int grid, int warps, size_t smem, const T* A, const T* B, T* C,
                            cudaStream_t s) {
  if (smem > 48 * 1024)
    VBG_CUDA(cudaFuncSetAttribute(spgemm_numeric_kernel<T, R>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)smem));
  spgemm_numeric_kernel<T, R><<<grid, warps * 32, smem, s>>>(x, A, B, C);
  return 0;
}

template <typename T>
static int launch_numeric(int r, const NumArgs& x, int grid, int warps, size_t smem, const T* A, const T* B, T* C,
                          cudaStream_t s) {
  switch (r) {
    case 1: return launch_numeric_r<T, 1>(x, grid, warps, smem, A, B, C, s);
    case 2: return launch_numeric_r<T, 2>(x, grid, warps, smem, A, B, C, s);
    case 3: return launch_numeric_r<T, 3>(x, grid, warps, smem, A, B, C, s);
    case 4: return launch_numeric_r<T, 4>(x, grid, warps, smem, A, B, C, s);
    case 5: return launch_numeric_r<T, 5>(x, grid, warps, smem, A, B, C, s);
    case 6: return launch_numeric_r<T, 6>(x, grid, warps, smem, A, B, C, s);
    case 7: return launch_numeric_r<T, 7>(x, grid, warps, smem, A, B, C, s);
    case 8: return launch_numeric_r<T, 8>(x, grid, warps, smem, A, B, C, s);
    default: return launch_numeric_r<T, 0>(x, grid, warps, smem, A, B, C, s);
  }
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

// Warp per row i of A: the symbolic table size of C's row i, 2 b + 1 with b
// the least of n, the sum of the lengths of the B rows k that A's row
// touches (common.hpp:600-616 sizes its tables by these two) and the span
// of the column range those B rows cover (their columns are sorted); -1 for
// an empty row.
__global__ void sym_need_kernel(int n, const int* __restrict__ a_rp, const int* __restrict__ a_ci,
                                const int* __restrict__ b_rp, const int* __restrict__ b_ci, int64_t* __restrict__ need) {
  const int lane = threadIdx.x & 31;
  const int warps = gridDim.x * (blockDim.x >> 5);
  for (int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); i < n; i += warps) {
    long long bound = 0;
    int lo = INT32_MAX, hi = -1;
    for (int p = a_rp[i] + lane; p < a_rp[i + 1]; p += 32) {
      const int k = a_ci[p];
      const int q0 = b_rp[k], q1 = b_rp[k + 1];
      if (q1 > q0) {
        bound += q1 - q0;
        lo = min(lo, b_ci[q0]);
        hi = max(hi, b_ci[q1 - 1]);
      }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      bound += __shfl_xor_sync(0xffffffffu, bound, off);
      lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, off));
      hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, off));
    }
    if (lane == 0) {
      const long long b = min(min(bound, (long long)n), (long long)hi - lo + 1);
      need[i] = bound == 0 ? -1 : 2 * b + 1;
    }
  }
}

// Thread per C row: its blocks and scalars.
__global__ void num_need_kernel(int n, const int* __restrict__ c_rp, const int64_t* __restrict__ c_off,
                                int64_t* __restrict__ out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int p0 = c_rp[i], p1 = c_rp[i + 1];
    out[2 * (size_t)i] = p1 - p0;
    out[2 * (size_t)i + 1] = c_off[p1] - c_off[p0];
  }
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
  DevBuf nA(s), nB(s), cnt(s), err(s), gtab(s), rows_dev(s);
  if ((rc = nA.ensure(std::max<int64_t>(A->nnzb, 1) * 8))) return rc;
  if ((rc = nB.ensure(std::max<int64_t>(B->nnzb, 1) * 8))) return rc;
  if ((rc = block_norms_dev(A, nA.as<double>(), s))) return rc;
  if ((rc = block_norms_dev(B, nB.as<double>(), s))) return rc;
  if ((rc = cnt.ensure((n + 1) * sizeof(int)))) return rc;
  if ((rc = err.ensure(16))) return rc;
  VBG_CUDA(cudaMemsetAsync(err.p, 0, 16, s));
  VBG_CUDA(cudaMemsetAsync(cnt.p, 0, (n + 1) * sizeof(int), s));
  const int serial_b = B->dup_cols ? 1 : 0;

  // symbolic table sizes, computed on the device (sym_need_kernel)
  std::vector<int64_t> need(n, -1);
  if (n) {
    DevBuf dneed(s);
    if ((rc = dneed.ensure(n * sizeof(int64_t)))) return rc;
    const int g = std::max(1, std::min((n + 7) / 8, sm_count() * 16));
    sym_need_kernel<<<g, 256, 0, s>>>(n, A->row_ptr.as<int>(), A->col_ind.as<int>(), B->row_ptr.as<int>(),
                                      B->col_ind.as<int>(), dneed.as<int64_t>());
    VBG_CUDA(cudaGetLastError());
    VBG_CUDA(cudaMemcpyAsync(need.data(), dneed.p, n * sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    VBG_CUDA(cudaStreamSynchronize(s));
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
  DevBuf d_crp(s), d_cci(s), scan_tmp(s);
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
  C->dup_cols = false;  // the symbolic phase lists distinct columns
  const size_t es = elem_size(C->dtype);
  if ((rc = C->vals.ensure(std::max<int64_t>(C->nnz, 1) * es, s))) return rc;
  DevBuf keep(s), prods(s);
  if ((rc = keep.ensure(std::max<int64_t>(cnnzb, 1)))) return rc;
  if ((rc = prods.ensure(16))) return rc;
  VBG_CUDA(cudaMemsetAsync(prods.p, 0, 16, s));

  // per C row: blocks and scalars (num_need_kernel)
  std::vector<int64_t> rowsz(2 * (size_t)n);
  if (n) {
    DevBuf drs(s);
    if ((rc = drs.ensure(2 * (size_t)n * sizeof(int64_t)))) return rc;
    num_need_kernel<<<std::max(1, std::min((n + 255) / 256, sm_count() * 8)), 256, 0, s>>>(
        n, C->row_ptr.as<int>(), C->blk_off.as<int64_t>(), drs.as<int64_t>());
    VBG_CUDA(cudaGetLastError());
    VBG_CUDA(cudaMemcpyAsync(rowsz.data(), drs.p, 2 * (size_t)n * sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    VBG_CUDA(cudaStreamSynchronize(s));
  }
  // Rows binned by the bytes of their region: table + accumulators in
  // shared memory when that fits kNumRowSmem, else (key < 0) the table
  // alone in global scratch.
  // Rows also grouped by block size R (every size <= 8), 0 otherwise.
  const bool small = std::max(A->max_bs, B->max_bs) <= 8;
  std::map<std::pair<int, int64_t>, std::vector<int>> nbins;
  for (int i = 0; i < n; ++i) {
    const int cnt = (int)rowsz[2 * (size_t)i];
    if (cnt == 0) continue;
    const int TT = num_table_size(cnt);
    const int64_t elems = rowsz[2 * (size_t)i + 1];
    const int64_t need = (int64_t)num_acc_offset(TT) + elems * (int64_t)es;
    const int rt = small ? A->h_bsz[i] : 0;
    if (need <= kNumRowSmem)
      nbins[{rt, next_pow2(std::max<int64_t>(need, 4096))}].push_back(i);
    else
      nbins[{rt, -(int64_t)next_pow2((int64_t)TT * 8)}].push_back(i);
  }
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
  {
    std::vector<int> all;
    all.reserve(n);
    for (auto& kv : nbins) all.insert(all.end(), kv.second.begin(), kv.second.end());
    if ((rc = rows_dev.ensure(std::max<size_t>(all.size(), 1) * sizeof(int)))) return rc;
    if (!all.empty())
      VBG_CUDA(cudaMemcpyAsync(rows_dev.p, all.data(), all.size() * sizeof(int), cudaMemcpyHostToDevice, s));
    size_t off = 0;
    const int wbytes = C->dtype == VBG_C128 ? num_warp_bytes<cplx>() : num_warp_bytes<double>();
    for (auto& kv : nbins) {
      NumArgs x = na;
      x.rows = rows_dev.as<int>() + off;
      x.nrows = (int)kv.second.size();
      off += kv.second.size();
      int grid;
      size_t smem;
      if (kv.first.second > 0) {
        x.region = (int)kv.first.second;
        smem = (size_t)kNumWarps * wbytes + x.region;
        grid = std::max(1, std::min(x.nrows, sm_count() * 16));
        x.gtab = nullptr;
      } else {
        x.region = (int)(-kv.first.second);
        smem = (size_t)kNumWarps * wbytes;
        grid = std::max(1, std::min(x.nrows, sm_count() * 4));
        if ((rc = gtab.ensure((size_t)grid * x.region))) return rc;
        x.gtab = gtab.as<char>();
      }
      if (C->dtype == VBG_C128)
        rc = launch_numeric<cplx>(kv.first.first, x, grid, kNumWarps, smem, A->vals.as<cplx>(), B->vals.as<cplx>(),
                                  C->vals.as<cplx>(), s);
      else
        rc = launch_numeric<double>(kv.first.first, x, grid, kNumWarps, smem, A->vals.as<double>(),
                                    B->vals.as<double>(), C->vals.as<double>(), s);
      if (rc) return rc;
      VBG_CUDA(cudaGetLastError());
    }
  }
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
