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
constexpr int kNumItem = 8;    // C blocks per numeric work item
constexpr int kPairBatch = 4;  // block pairs whose operands are loaded together
constexpr int kNumWarpsCta = 8;  // warps of a numeric CTA
constexpr long long kOffMask = (1ll << 56) - 1;  // pair list: offset bits below the inner size

struct SymArgs {
  const int* a_rp;
  const int* a_ci;
  const double* nA;
  const int* b_rp;
  const int* b_ci;
  const double* nB;
  double thr;
  int serial_lanes;   // B has duplicate columns in a row: one lane at a time
  int upper;          // only block columns >= the row (the upper block triangle)
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
        if (lane < width && b < b1 && !(a.upper && a.b_ci[b] < row)) {
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
  const int* bt_ptr;    // B's column view: entry range of each block column,
  const int* bt_row;    // the row k of each entry (ascending within a column)
  const int* bt_slot;   // and its slot
  const int64_t* b_off;
  const double* nB;
  const int* bsz;
  const int* c_ci;
  const int64_t* c_off;
  const int4* items;    // work items {row, first C slot, C slots} of one row size
  int dup;              // B holds some block column twice in a row
  int nitems;
  double thr;
  unsigned char* keep;  // per C slot
  unsigned long long* products;
};

__device__ __forceinline__ double sq_mag(double v) { return __dmul_rn(v, v); }
__device__ __forceinline__ double sq_mag(float v) { return __dmul_rn((double)v, (double)v); }
__device__ __forceinline__ double sq_mag(cplx v) { return fma(v.re, v.re, __dmul_rn(v.im, v.im)); }

// D = A B + C for one 8 x 8 x 4 FP64 tile (mma.sync m8n8k4, row.col): lane l
// holds A(l / 4, l % 4), B(l % 4, l / 4) and C(l / 4, 2 (l % 4) + {0, 1}).
__device__ __forceinline__ void dmma_884(double& c0, double& c1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}

// Accumulator of one C block C_ij (r x c, row-major) held by a warp.  Blocks
// of at most 8 x 8 (R != 0) live in registers in the layout of the m8n8k4 C
// fragment: lane l holds (l / 4, 2 (l % 4) + {0, 1}).  Real blocks multiply on
// the FP64 tensor cores, complex ones with scalar fused multiply-adds; blocks
// over 8 (R == 0) accumulate in their slice of C itself, lanes over the
// elements.
template <typename T, int R>
struct BlockAcc {
  T v0, v1;
  __device__ __forceinline__ void zero(T* cp, int r, int c, int lane) {
    v0 = v1 = zero_s<T>();
    if constexpr (R == 0)
      for (int e = lane; e < r * c; e += 32) cp[e] = zero_s<T>();
  }
  // Fragments of one pair for the tensor-core path (real, R != 0): the A
  // and B elements this lane holds for the two k-halves, zero outside the
  // blocks.
  struct Frag {
    double a0, a1, b0, b1;
  };
  // B element indices of this lane for a C block of c columns (the B block
  // is inner x c row-major; valid when the lane's column gq < c).
  int bi0 = 0, bi1 = 0;
  bool bcol = false;
  __device__ __forceinline__ void begin(int c, int lane) {
    const int gq = lane >> 2, t4 = lane & 3;
    bi0 = t4 * c + gq;
    bi1 = (t4 + 4) * c + gq;
    bcol = gq < c;
  }
  __device__ __forceinline__ void load_pre(Frag& f, const T* __restrict__ ap, const T* __restrict__ bp, int inner,
                                           int lane) const {
    const int gq = lane >> 2, t4 = lane & 3;
    const double* a = reinterpret_cast<const double*>(ap);
    const double* b = reinterpret_cast<const double*>(bp);
    const int ai = gq * inner + t4;
    f.a0 = (gq < R && t4 < inner) ? a[ai] : 0.0;
    f.b0 = (bcol && t4 < inner) ? b[bi0] : 0.0;
    f.a1 = (gq < R && t4 + 4 < inner) ? a[ai + 4] : 0.0;
    f.b1 = (bcol && t4 + 4 < inner) ? b[bi1] : 0.0;
  }
  __device__ __forceinline__ void mma(const Frag& f, int inner) {
    double x0 = v0, x1 = v1;
    dmma_884(x0, x1, f.a0, f.b0);
    if (inner > 4) dmma_884(x0, x1, f.a1, f.b1);
    v0 = x0;
    v1 = x1;
  }
  // C_ij += A_ik (r x inner) B_kj (inner x c), each element a fused
  // multiply-add chain over the inner index in order (R == 0 and complex),
  // or two m8n8k4 steps over it (real).
  __device__ __forceinline__ void mac(const T* __restrict__ ap, const T* __restrict__ bp, T* cp, int r, int inner,
                                      int c, int lane) {
    const int gq = lane >> 2, t4 = lane & 3;
    if constexpr (R != 0 && sizeof(T) == sizeof(double)) {
      const double* a = reinterpret_cast<const double*>(ap);
      const double* b = reinterpret_cast<const double*>(bp);
      const double a0 = (gq < R && t4 < inner) ? a[gq * inner + t4] : 0.0;
      const double b0 = (t4 < inner && gq < c) ? b[t4 * c + gq] : 0.0;
      double x0 = v0, x1 = v1;
      dmma_884(x0, x1, a0, b0);
      if (inner > 4) {
        const double a1 = (gq < R && t4 + 4 < inner) ? a[gq * inner + t4 + 4] : 0.0;
        const double b1 = (t4 + 4 < inner && gq < c) ? b[(t4 + 4) * c + gq] : 0.0;
        dmma_884(x0, x1, a1, b1);
      }
      v0 = x0;
      v1 = x1;
    } else if constexpr (R != 0) {
      if (gq < R) {
        const int u = 2 * t4;
#pragma unroll
        for (int q = 0; q < 8; ++q)
          if (q < inner) {
            const T x = ap[gq * inner + q];
            if (u < c) v0 = fma_s(x, bp[q * c + u], v0);
            if (u + 1 < c) v1 = fma_s(x, bp[q * c + u + 1], v1);
          }
      }
    } else {
      for (int e = lane; e < r * c; e += 32) {
        const int t = e / c, u = e - t * c;
        T v = cp[e];
        for (int q = 0; q < inner; ++q) v = fma_s(ap[t * inner + q], bp[q * c + u], v);
        cp[e] = v;
      }
    }
  }
  // Writes the block (register layouts) and returns its squared Frobenius
  // norm, summed over the warp.
  __device__ __forceinline__ double finish(T* cp, int r, int c, int lane) {
    double sq = 0.0;
    if constexpr (R != 0) {
      const int gq = lane >> 2, u = 2 * (lane & 3);
      if (gq < r) {
        if (u < c) {
          cp[gq * c + u] = v0;
          sq = sq_mag(v0);
        }
        if (u + 1 < c) {
          cp[gq * c + u + 1] = v1;
          sq = __dadd_rn(sq, sq_mag(v1));
        }
      }
    } else {
      __syncwarp();
      for (int e = lane; e < r * c; e += 32) sq = __dadd_rn(sq, sq_mag(cp[e]));
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) sq += __shfl_xor_sync(0xffffffffu, sq, off);
    return sq;
  }
};

// Numeric phase, inner-product form: a warp takes a work item -- up to
// kNumItem consecutive C blocks of one block row i, all rows of the launch of
// block size R (R = 0: any size) -- and computes each C_ij in turn as the
// sum over k of A_ik B_kj, k running over the block columns of A's row i
// that B's column j also holds, in increasing order (A's slot order).  For
// 32 A slots at a time the lanes find their k in B's column list by binary
// search; a pair is skipped when |A_ik| |B_kj| < threshold / max(1,
// nnzb(A row i)) (vbcsr.hpp:372, :386).  The matches are taken one at a time
// in lane order (a column holding k more than once gives several pairs, in
// slot order).  The Frobenius norm of each finished block gives the filter's
// keep flag.
template <typename T, int R>
__global__ void __launch_bounds__(kNumWarpsCta * 32, 3) spgemm_numeric_kernel(NumArgs a, const T* __restrict__ A,
                                                             const T* __restrict__ B, T* __restrict__ C) {
  __shared__ longlong2 plists[kNumWarpsCta][32];
  const int lane = threadIdx.x & 31;
  const int nwarps = gridDim.x * (blockDim.x >> 5);
  longlong2* plist = plists[threadIdx.x >> 5];
  unsigned long long prods = 0;
  for (int w = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); w < a.nitems; w += nwarps) {
    const int4 it = a.items[w];
    const int row = it.x;
    const int a0 = a.a_rp[row], a1 = a.a_rp[row + 1];
    const double row_eps = a.thr / (double)max(1, a1 - a0);
    const int r = R ? R : a.bsz[row];
    for (int p = it.y; p < it.y + it.z; ++p) {
      const int j = a.c_ci[p];
      const int c = a.bsz[j];
      const int q0 = a.bt_ptr[j], q1 = a.bt_ptr[j + 1];
      T* cp = C + a.c_off[p];
      BlockAcc<T, R> acc;
      acc.zero(cp, r, c, lane);
      acc.begin(c, lane);
      for (int base = a0; base < a1; base += 32) {
        const int as = base + lane;
        const int k = as < a1 ? a.a_ci[as] : -1;
        int lo = q0, hi = q1;
        while (lo < hi) {
          const int mid = (lo + hi) >> 1;
          if (a.bt_row[mid] < k) lo = mid + 1;
          else hi = mid;
        }
        int cnt = 0;
        if (k >= 0)
          while (lo + cnt < q1 && a.bt_row[lo + cnt] == k) ++cnt;
        // this lane's pair (its first match): offsets loaded by all lanes at once
        const int bs1 = cnt > 0 ? a.bt_slot[lo] : 0;
        const bool pass1 = cnt == 1 && !(a.nA[as] * a.nB[bs1] < row_eps);
        const int64_t aoff = cnt > 0 ? a.a_off[as] : 0;
        const int64_t boff = cnt > 0 ? a.b_off[bs1] : 0;
        const int inn = cnt > 0 ? a.bsz[k] : 0;
        if (!a.dup) {
          // distinct columns: at most one match per lane; the kept pairs in
          // lane order, up to kPairBatch at a time with all their fragment
          // loads issued before the multiply chain
          // The pair list goes through shared memory: lane order, the A
          // offset with the inner size in its top byte, then the B offset.
          const unsigned m = __ballot_sync(0xffffffffu, pass1);
          const int np = __popc(m);
          if (pass1)
            plist[__popc(m & ((1u << lane) - 1u))] =
                make_longlong2((long long)aoff | ((long long)inn << 56), (long long)boff);
          __syncwarp();
          for (int b0 = 0; b0 < np; b0 += kPairBatch) {
            if constexpr (R != 0 && sizeof(T) == sizeof(double)) {
              typename BlockAcc<T, R>::Frag f[kPairBatch];
              int fin[kPairBatch];
#pragma unroll
              for (int b = 0; b < kPairBatch; ++b) {
                fin[b] = 0;
                if (b0 + b < np) {
                  const longlong2 e = plist[b0 + b];
                  fin[b] = (int)(e.x >> 56);
                  acc.load_pre(f[b], A + (e.x & kOffMask), B + e.y, fin[b], lane);
                }
              }
#pragma unroll
              for (int b = 0; b < kPairBatch; ++b)
                if (b0 + b < np) acc.mma(f[b], fin[b]);
            } else {
#pragma unroll
              for (int b = 0; b < kPairBatch; ++b)
                if (b0 + b < np) {
                  const longlong2 e = plist[b0 + b];
                  acc.mac(A + (e.x & kOffMask), B + e.y, cp, r, (int)(e.x >> 56), c, lane);
                }
            }
          }
          prods += np;
          __syncwarp();
        } else {
          // a column may hold k more than once: every match, in order
          unsigned m = __ballot_sync(0xffffffffu, cnt > 0);
          while (m) {
            const int src = __ffs(m) - 1;
            m &= m - 1;
            const int s_as = __shfl_sync(0xffffffffu, as, src);
            const int s_lo = __shfl_sync(0xffffffffu, lo, src);
            const int s_cnt = __shfl_sync(0xffffffffu, cnt, src);
            const int s_inn = __shfl_sync(0xffffffffu, inn, src);
            const T* ap = A + a.a_off[s_as];
            for (int t = 0; t < s_cnt; ++t) {
              const int bs = a.bt_slot[s_lo + t];
              if (a.nA[s_as] * a.nB[bs] < row_eps) continue;
              acc.mac(ap, B + a.b_off[bs], cp, r, s_inn, c, lane);
              ++prods;
            }
          }
        }
      }
      const double sq = acc.finish(cp, r, c, lane);
      if (lane == 0) a.keep[p] = (a.thr <= 0.0 || sqrt(sq) >= a.thr) ? 1 : 0;
    }
  }
  if (lane == 0 && prods) atomicAdd(a.products, prods);
}

// FP32 product results into the FP64 values of C.
__global__ void widen_f32_kernel(const float* __restrict__ in, double* __restrict__ out, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = (double)in[i];
}

template <typename T, int R>
static int launch_numeric_r(const NumArgs& x, const T* A, const T* B, T* C, cudaStream_t s) {
  const int grid = std::max(1, std::min((x.nitems + kNumWarpsCta - 1) / kNumWarpsCta, sm_count() * 16));
  spgemm_numeric_kernel<T, R><<<grid, kNumWarpsCta * 32, 0, s>>>(x, A, B, C);
  return 0;
}

template <typename T>
static int launch_numeric(int r, const NumArgs& x, const T* A, const T* B, T* C, cudaStream_t s) {
  switch (r) {
    case 1: return launch_numeric_r<T, 1>(x, A, B, C, s);
    case 2: return launch_numeric_r<T, 2>(x, A, B, C, s);
    case 3: return launch_numeric_r<T, 3>(x, A, B, C, s);
    case 4: return launch_numeric_r<T, 4>(x, A, B, C, s);
    case 5: return launch_numeric_r<T, 5>(x, A, B, C, s);
    case 6: return launch_numeric_r<T, 6>(x, A, B, C, s);
    case 7: return launch_numeric_r<T, 7>(x, A, B, C, s);
    case 8: return launch_numeric_r<T, 8>(x, A, B, C, s);
    default: return launch_numeric_r<T, 0>(x, A, B, C, s);
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
// an empty row.  `upper`: only columns >= i are inserted, so the span starts
// at i at the earliest (-1 when every column lies below the row).
__global__ void sym_need_kernel(int n, const int* __restrict__ a_rp, const int* __restrict__ a_ci,
                                const int* __restrict__ b_rp, const int* __restrict__ b_ci, int upper,
                                int64_t* __restrict__ need) {
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
      if (upper) lo = max(lo, i);
      const long long span = (long long)hi - lo + 1;
      const long long b = min(min(bound, (long long)n), span);
      need[i] = (bound == 0 || span <= 0) ? -1 : 2 * b + 1;
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

// The thresholded product C = A B; with `upper`, only its block columns at
// or above each row (the symbolic phase skips the others, and the numeric
// phase follows C's pattern).
static int spgemm_run(const vbg_matrix* A, const vbg_matrix* B, double thr, int upper, vbg_matrix** Cout,
                      int64_t* stats, cudaStream_t s, int precision = VBG_PREC_F64) {
  VBG_CHECK(A && B && Cout, VBG_E_ARG, "null argument");
  VBG_CHECK(A->dtype == B->dtype, VBG_E_ARG, "A and B must have the same dtype");
  VBG_CHECK(precision == VBG_PREC_F64 || (precision == VBG_PREC_F32 && A->dtype == VBG_F64), VBG_E_ARG,
            "precision must be VBG_PREC_F64, or VBG_PREC_F32 for real matrices");
  VBG_CHECK(A->n == B->n && A->h_bsz == B->h_bsz, VBG_E_ARG, "spmm: A's columns and B's rows differ");
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
  // page-locked staging of this thread's calls (each use completes before
  // the call returns)
  thread_local HostBuf h_rows, h_items;
  std::vector<int64_t> need(n, -1);
  if (n) {
    DevBuf dneed(s);
    if ((rc = dneed.ensure(n * sizeof(int64_t)))) return rc;
    if ((rc = h_rows.ensure(n * sizeof(int64_t)))) return rc;
    const int g = std::max(1, std::min((n + 7) / 8, sm_count() * 16));
    sym_need_kernel<<<g, 256, 0, s>>>(n, A->row_ptr.as<int>(), A->col_ind.as<int>(), B->row_ptr.as<int>(),
                                      B->col_ind.as<int>(), upper, dneed.as<int64_t>());
    VBG_CUDA(cudaGetLastError());
    VBG_CUDA(cudaMemcpyAsync(h_rows.p, dneed.p, n * sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    VBG_CUDA(cudaStreamSynchronize(s));
    std::memcpy(need.data(), h_rows.p, n * sizeof(int64_t));
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
  sa.upper = upper;
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
  const int64_t* rowsz = nullptr;  // in h_rows
  if (n) {
    DevBuf drs(s);
    if ((rc = drs.ensure(2 * (size_t)n * sizeof(int64_t)))) return rc;
    if ((rc = h_rows.ensure(2 * (size_t)n * sizeof(int64_t)))) return rc;
    num_need_kernel<<<std::max(1, std::min((n + 255) / 256, sm_count() * 8)), 256, 0, s>>>(
        n, C->row_ptr.as<int>(), C->blk_off.as<int64_t>(), drs.as<int64_t>());
    VBG_CUDA(cudaGetLastError());
    VBG_CUDA(cudaMemcpyAsync(h_rows.p, drs.p, 2 * (size_t)n * sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    VBG_CUDA(cudaStreamSynchronize(s));
    rowsz = h_rows.as<int64_t>();
  }
  // Work items {row, first C slot, C slots <= kNumItem}, grouped by the row's
  // block size (all sizes <= 8; else one group, R = 0).
  const bool small = std::max(A->max_bs, B->max_bs) <= 8;
  std::vector<int64_t> gcount(9, 0);  // items per group (row block size, 0 = any)
  for (int i = 0; i < n; ++i)
    gcount[small ? A->h_bsz[i] : 0] += (rowsz[2 * (size_t)i] + kNumItem - 1) / kNumItem;
  std::vector<int64_t> gstart(10, 0);
  for (int g = 0; g < 9; ++g) gstart[g + 1] = gstart[g] + gcount[g];
  const int64_t nitems = gstart[9];
  if ((rc = h_items.ensure(std::max<int64_t>(nitems, 1) * sizeof(int4)))) return rc;
  {
    int4* it = h_items.as<int4>();
    std::vector<int64_t> fill(gstart.begin(), gstart.end() - 1);
    int64_t first = 0;
    for (int i = 0; i < n; ++i) {
      const int cnt = (int)rowsz[2 * (size_t)i];
      int64_t& f = fill[small ? A->h_bsz[i] : 0];
      for (int o = 0; o < cnt; o += kNumItem) it[f++] = make_int4(i, (int)(first + o), std::min(kNumItem, cnt - o), 0);
      first += cnt;
    }
  }
  if ((rc = build_csc_dev(B, s))) return rc;
  NumArgs na{};
  na.a_rp = A->row_ptr.as<int>();
  na.a_ci = A->col_ind.as<int>();
  na.a_off = A->blk_off.as<int64_t>();
  na.nA = nA.as<double>();
  na.bt_ptr = B->csc_ptr.as<int>();
  na.bt_row = B->csc_row.as<int>();
  na.bt_slot = B->csc_slot.as<int>();
  na.b_off = B->blk_off.as<int64_t>();
  na.nB = nB.as<double>();
  na.bsz = A->bsz.as<int>();
  na.c_ci = C->col_ind.as<int>();
  na.c_off = C->blk_off.as<int64_t>();
  na.thr = thr;
  na.dup = B->dup_cols ? 1 : 0;
  na.keep = keep.as<unsigned char>();
  na.products = prods.as<unsigned long long>();
  {
    DevBuf items(s), c32(s);
    if ((rc = items.ensure(std::max<int64_t>(nitems, 1) * sizeof(int4)))) return rc;
    if (nitems) VBG_CUDA(cudaMemcpyAsync(items.p, h_items.p, nitems * sizeof(int4), cudaMemcpyHostToDevice, s));
    const bool f32 = precision == VBG_PREC_F32;
    if (f32) {
      // FP32 operands (the shadows) and FP32 accumulation; the block norms,
      // the skip and keep rules stay FP64
      if ((rc = ensure_vals32(A, s))) return rc;
      if ((rc = ensure_vals32(B, s))) return rc;
      if ((rc = c32.ensure(std::max<int64_t>(C->nnz, 1) * sizeof(float)))) return rc;
    }
    for (int g = 0; g < 9; ++g) {
      if (!gcount[g]) continue;
      NumArgs x = na;
      x.items = items.as<int4>() + gstart[g];
      x.nitems = (int)gcount[g];
      if (C->dtype == VBG_C128)
        rc = launch_numeric<cplx>(g, x, A->vals.as<cplx>(), B->vals.as<cplx>(), C->vals.as<cplx>(), s);
      else if (f32)
        rc = launch_numeric<float>(g, x, A->vals32.as<float>(), B->vals32.as<float>(), c32.as<float>(), s);
      else
        rc = launch_numeric<double>(g, x, A->vals.as<double>(), B->vals.as<double>(), C->vals.as<double>(), s);
      if (rc) return rc;
      VBG_CUDA(cudaGetLastError());
    }
    if (f32 && C->nnz) {
      const int g = (int)std::max<int64_t>(1, std::min<int64_t>((C->nnz + 255) / 256, (int64_t)sm_count() * 16));
      widen_f32_kernel<<<g, 256, 0, s>>>(c32.as<float>(), C->vals.as<double>(), C->nnz);
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

extern "C" int vbg_spgemm(const vbg_matrix* A, const vbg_matrix* B, double thr, vbg_matrix** Cout, int64_t* stats,
                          void* stream) {
  return spgemm_run(A, B, thr, 0, Cout, stats, as_stream(stream));
}

extern "C" int vbg_spgemm_ex(const vbg_matrix* A, const vbg_matrix* B, double thr, int precision, int hermitian,
                             vbg_matrix** Cout, int64_t* stats, void* stream) {
  cudaStream_t s = as_stream(stream);
  vbg_matrix* C = nullptr;
  int rc = spgemm_run(A, B, thr, hermitian ? 1 : 0, &C, stats, s, precision);
  if (rc) return rc;
  std::unique_ptr<vbg_matrix> keep(C);
  if (hermitian) {
    if ((rc = complete_hermitian_dev(C, s))) return rc;
    if (stats) stats[1] = C->nnzb;
  }
  *Cout = keep.release();
  return 0;
}

extern "C" int vbg_spgemm_hermitian(const vbg_matrix* A, const vbg_matrix* B, double thr, vbg_matrix** Cout,
                                    int64_t* stats, void* stream) {
  cudaStream_t s = as_stream(stream);
  vbg_matrix* U = nullptr;
  int rc = spgemm_run(A, B, thr, 1, &U, stats, s);
  if (rc) return rc;
  std::unique_ptr<vbg_matrix> keep(U);
  if ((rc = complete_hermitian_dev(U, s))) return rc;
  if (stats) stats[1] = U->nnzb;
  *Cout = keep.release();
  return 0;
}
