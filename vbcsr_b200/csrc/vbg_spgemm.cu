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
#include <type_traits>
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
constexpr int kWinCap = 1024;    // numeric: entries of a warp's window table of A's row
constexpr int kRowStageCap = 8192;  // numeric row kernel: A row values staged in shared memory (64 KB)

// Pair gates.  kGateSum is the plain product (symbolic: keep j iff
// sum_k |A_ik||B_kj| > threshold; numeric: skip a pair below threshold /
// max(1, n_A)).  The others are the fused triple products' per-row gates
// (ops/spmm/rarh.hpp, rhar.hpp, square_polynomial.hpp): a pair
// (i,k)(k,j) reaches C's row only when |L_ik||R_kj| >= eps, and every column
// a pair reaches is kept by the symbolic phase:
//   kGateStage1  eps = thr / (2 max(1, n_L) |R row k| max|A|)   (T = L B)
//   kGateStage2  eps = thr / (2 n_L), |L_ik| the stage-one bound  (C = T A)
//   kGatePoly    eps = thr / max(1, n_L), 0 for an all-zero A      (A A)
// with n_L the left operand's blocks in row i; every eps is 0 for thr <= 0.
constexpr int kGateSum = 0;
constexpr int kGateStage1 = 1;
constexpr int kGateStage2 = 2;
constexpr int kGatePoly = 3;

__host__ __device__ inline double gate_eps(int mode, double thr, double amax, int nl, int nb) {
  if (mode == kGateStage1)
    return (thr > 0.0 && amax > 0.0 && nb > 0) ? thr / (2.0 * (double)(nl > 1 ? nl : 1) * (double)nb * amax) : 0.0;
  if (mode == kGateStage2) return (thr > 0.0 && nl > 0) ? thr / (2.0 * (double)nl) : 0.0;
  if (mode == kGatePoly) return (thr > 0.0 && amax > 0.0) ? thr / (double)(nl > 1 ? nl : 1) : 0.0;
  return thr / (double)(nl > 1 ? nl : 1);
}

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
  int mode;           // kGate*
  const double* amax; // gated modes: the largest block norm of A (device)
  int self_cols;      // kGatePoly: A's own columns (>= the row) and the diagonal join every row
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
    const int nl = a.a_rp[row + 1] - a.a_rp[row];
    const double amax = a.mode != kGateSum ? *a.amax : 0.0;
    if (a.self_cols) {
      // the c1 A and c0 I terms reach A's own columns and the diagonal
      for (int as = a.a_rp[row] + lane; as <= a.a_rp[row + 1]; as += 32) {
        const int j = as < a.a_rp[row + 1] ? a.a_ci[as] : row;
        if (a.upper && j < row) continue;
        int h = j & mask;
        for (int probes = 0;; ++probes) {
          int k = keys[h];
          if (k == kEmpty) k = atomicCAS(&keys[h], kEmpty, j);
          if (k == kEmpty || k == j) {
            vals[h] = 1.0;
            break;
          }
          h = (h + 1) & mask;
          if (probes > T) {
            atomicExch(a.err, 1);
            break;
          }
        }
      }
      __syncwarp();
    }
    for (int as = a.a_rp[row]; as < a.a_rp[row + 1]; ++as) {
      const int kk = a.a_ci[as];
      const double na = a.nA[as];
      const int b0 = a.b_rp[kk], b1 = a.b_rp[kk + 1];
      const double eps = a.mode != kGateSum ? gate_eps(a.mode, a.thr, amax, nl, b1 - b0) : 0.0;
      const int width = a.serial_lanes ? 1 : 32;
      for (int bc = b0; bc < b1; bc += width) {
        const int b = bc + lane;
        const double v = (lane < width && b < b1) ? __dmul_rn(na, a.nB[b]) : 0.0;
        // gated modes: a pair below its gate does not reach the row
        if (lane < width && b < b1 && !(a.upper && a.b_ci[b] < row) && (a.mode == kGateSum || !(v < eps))) {
          const int j = a.b_ci[b];
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
    // kept columns: sum > threshold (common.hpp:664); gated: every column reached
    int base_pos = 0;
    for (int h0 = 0; h0 < T; h0 += 32) {
      const int h = h0 + lane;
      const bool kept = keys[h] != kEmpty && (a.mode != kGateSum || vals[h] > a.thr);
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
  const int4* items;    // work items {row, first C slot, C slots}, rows in class order
  const int* item_start;  // first item of each class-ordered row (exclusive scan, n + 1)
  int w0, w1;           // this launch: class-ordered rows [w0, w1), items [item_start[w0], item_start[w1])
  int dup;              // B holds some block column twice in a row
  int window;           // neither A nor B holds a block column twice in a row: A rows may be mapped
  double thr;
  unsigned char* keep;  // per C slot
  unsigned long long* products;
  int mode;             // kGate*
  const double* amax;   // gated modes: the largest block norm of A (device)
  const int* b_rp;      // B's row pointers (kGateStage1 divides by B's row lengths)
  double* bound_out;    // per C slot: the sum of the norms of its kept pairs (nullptr: not wanted)
  int drop;             // keep flags from the finished blocks' norms (else every block is kept)
  const int* perm;      // row kernel: C's rows in class order
  const int* c_rp;      // row kernel: C's row pointers
  int row_cap;          // row kernel: A row values staged in shared memory up to this many
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
// that B's column j also holds, in increasing order.  A pair is skipped when
// |A_ik| |B_kj| < threshold / max(1, nnzb(A row i)) (vbcsr.hpp:372, :386).
// The Frobenius norm of each finished block gives the filter's keep flag.
//
// Finding the pairs.  When the block columns of A's row i span at most
// kWinCap (banded and lattice orderings), the warp maps
// the row once per work item into a window table in shared memory (block
// column k -> A slot); for each C block the lanes then walk B's column j
// (its rows k ascending, coalesced) and look k up in the table: one
// shared-memory load per entry.  Other rows keep the general search: for 32
// of A's slots at a time the lanes find their k in B's column list by binary
// search (a column holding k more than once gives several pairs, in slot
// order).  Either way the kept pairs of 32 candidates go through a list in
// shared memory, kPairBatch at a time with all their operand loads issued
// before the multiply chain.
// GATED: the fused products' gate modes and pair-norm bounds (kGate* other
// than kGateSum); the plain product compiles without them.
// One C block C_ij (slot p; its row has r scalar rows) of the numeric phase: the
// kept pairs of A's row and B's column j, multiplied and written, the keep
// flag (and with GATED the pair-norm bound) stored.  span > 0: A's row is
// mapped in wtab (column kmin + d -> slot).  A's value at offset o is A[o]
// (the row kernel passes a base that puts A's row in shared memory).
template <typename T, int R, bool GATED>
__device__ __forceinline__ void numeric_block(const NumArgs& a, const T* __restrict__ A, const T* __restrict__ B,
                                              T* __restrict__ C, int p, int r, int a0, int a1, int kmin, int span,
                                              const int* wtab, longlong2* plist, int lane, double row_eps,
                                              double amax, unsigned long long& prods) {
  const int j = a.c_ci[p];
  const int c = a.bsz[j];
  const int q0 = a.bt_ptr[j], q1 = a.bt_ptr[j + 1];
  T* cp = C + a.c_off[p];
  BlockAcc<T, R> acc;
  acc.zero(cp, r, c, lane);
  acc.begin(c, lane);
  double bsum = 0.0;  // this lane's kept pair norms (bound_out)
  // rounds of 32 candidates: entries of B's column j (window table) or
  // slots of A's row i (search)
  const int ncand = span > 0 ? q1 - q0 : a1 - a0;
  for (int base = 0; base < ncand; base += 32) {
    bool pass = false;
    int64_t aoff = 0, boff = 0;
    int inn = 0;
    if (span > 0) {
      // k outside A's row range or absent from it gives no pair
      const int t = q0 + base + lane;
      const int k = t < q1 ? a.bt_row[t] : -1;
      const unsigned d = (unsigned)(k - kmin);
      const int as = (k >= 0 && d < (unsigned)span) ? wtab[d] : -1;
      const int bs = as >= 0 ? a.bt_slot[t] : 0;
      const double eps = GATED && a.mode == kGateStage1 && as >= 0
                             ? gate_eps(kGateStage1, a.thr, amax, a1 - a0, a.b_rp[k + 1] - a.b_rp[k])
                             : row_eps;
      const double pn = as >= 0 ? a.nA[as] * a.nB[bs] : 0.0;
      pass = as >= 0 && !(pn < eps);
      if (pass) {
        aoff = a.a_off[as];
        inn = a.bsz[k];
        boff = a.b_off[bs];
        if constexpr (GATED) bsum += pn;
      }
    } else {
      const int as = a0 + base + lane;
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
      if (a.dup) {
        // a column may hold k more than once: every match, in order
        unsigned m = __ballot_sync(0xffffffffu, cnt > 0);
        const int kin = cnt > 0 ? a.bsz[k] : 0;
        while (m) {
          const int src = __ffs(m) - 1;
          m &= m - 1;
          const int s_as = __shfl_sync(0xffffffffu, as, src);
          const int s_lo = __shfl_sync(0xffffffffu, lo, src);
          const int s_cnt = __shfl_sync(0xffffffffu, cnt, src);
          const int s_inn = __shfl_sync(0xffffffffu, kin, src);
          const T* ap = A + a.a_off[s_as];
          const int s_k = a.a_ci[s_as];
          const double eps = GATED && a.mode == kGateStage1
                                 ? gate_eps(kGateStage1, a.thr, amax, a1 - a0, a.b_rp[s_k + 1] - a.b_rp[s_k])
                                 : row_eps;
          for (int t = 0; t < s_cnt; ++t) {
            const int bs = a.bt_slot[s_lo + t];
            const double pn = a.nA[s_as] * a.nB[bs];
            if (pn < eps) continue;
            acc.mac(ap, B + a.b_off[bs], cp, r, s_inn, c, lane);
            if (GATED && lane == 0) bsum += pn;
            ++prods;
          }
        }
        continue;
      }
      // distinct columns: at most one match per lane
      const int bs1 = cnt > 0 ? a.bt_slot[lo] : 0;
      const double eps = GATED && a.mode == kGateStage1 && cnt > 0
                             ? gate_eps(kGateStage1, a.thr, amax, a1 - a0, a.b_rp[k + 1] - a.b_rp[k])
                             : row_eps;
      const double pn = cnt == 1 ? a.nA[as] * a.nB[bs1] : 0.0;
      pass = cnt == 1 && !(pn < eps);
      if (pass) {
        aoff = a.a_off[as];
        inn = a.bsz[k];
        boff = a.b_off[bs1];
        if constexpr (GATED) bsum += pn;
      }
    }
    // The kept pairs in lane order go through shared memory: the A
    // offset with the inner size in its top byte, then the B offset.
    const unsigned m = __ballot_sync(0xffffffffu, pass);
    const int np = __popc(m);
    if (pass)
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
  }
  const double sq = acc.finish(cp, r, c, lane);
  if (GATED && a.bound_out) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) bsum += __shfl_xor_sync(0xffffffffu, bsum, off);
    if (lane == 0) a.bound_out[p] = bsum;
  }
  if (lane == 0) a.keep[p] = ((GATED && !a.drop) || a.thr <= 0.0 || sqrt(sq) >= a.thr) ? 1 : 0;
}

template <typename T, int R, bool GATED = false>
__global__ void __launch_bounds__(kNumWarpsCta * 32, 3) spgemm_numeric_kernel(NumArgs a, const T* __restrict__ A,
                                                             const T* __restrict__ B, T* __restrict__ C) {
  __shared__ longlong2 plists[kNumWarpsCta][32];
  __shared__ int wtabs[kNumWarpsCta][kWinCap];
  const int lane = threadIdx.x & 31;
  const int nwarps = gridDim.x * (blockDim.x >> 5);
  longlong2* plist = plists[threadIdx.x >> 5];
  int* wtab = wtabs[threadIdx.x >> 5];
  unsigned long long prods = 0;
  const int i0 = a.item_start[a.w0], i1 = a.item_start[a.w1];
  for (int w = i0 + blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); w < i1; w += nwarps) {
    const int4 it = a.items[w];
    const int row = it.x;
    const int a0 = a.a_rp[row], a1 = a.a_rp[row + 1];
    const double amax = GATED ? *a.amax : 0.0;
    const double row_eps = gate_eps(GATED ? a.mode : kGateSum, a.thr, amax, a1 - a0, 0);  // kGateStage1: per pair below
    const int r = R ? R : a.bsz[row];
    // window table of A's row: slot of each block column k in [kmin, kmin + span)
    int kmin = 0, span = 0;
    if (a.window && a1 > a0) {
      int lo = INT32_MAX, hi = -1;
      for (int as = a0 + lane; as < a1; as += 32) {
        const int k = a.a_ci[as];
        lo = min(lo, k);
        hi = max(hi, k);
      }
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) {
        lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, off));
        hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, off));
      }
      if (hi - lo < kWinCap) {
        kmin = lo;
        span = hi - lo + 1;
        __syncwarp();  // the previous item's lookups are done
        for (int t = lane; t < span; t += 32) wtab[t] = -1;
        __syncwarp();
        for (int as = a0 + lane; as < a1; as += 32) wtab[a.a_ci[as] - kmin] = as;
        __syncwarp();
      }
    }
    for (int p = it.y; p < it.y + it.z; ++p)
      numeric_block<T, R, GATED>(a, A, B, C, p, r, a0, a1, kmin, span, wtab, plist, lane, row_eps, amax, prods);
  }
  if (lane == 0 && prods) atomicAdd(a.products, prods);
}

// Numeric phase, a CTA per C row (FP64 tensor-core path, A and B without
// repeated block columns): the row's A values (contiguous in A) are copied
// into shared memory once and its window table is built once, then the
// CTA's warps take the row's C blocks in turn and read A's fragments from
// shared memory -- only B's blocks come from L2.  Rows of A longer than
// row_cap values read A from global memory as the item kernel does.
template <typename T, int R, bool GATED>
__global__ void __launch_bounds__(kNumWarpsCta * 32, 3) spgemm_numeric_row_kernel(NumArgs a, const T* __restrict__ A,
                                                                 const T* __restrict__ B, T* __restrict__ C) {
  extern __shared__ __align__(16) unsigned char srow_raw[];
  T* srow = reinterpret_cast<T*>(srow_raw);
  __shared__ longlong2 plists[kNumWarpsCta][32];
  __shared__ int wtab[kWinCap];
  __shared__ int s_lo, s_hi;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  longlong2* plist = plists[warp];
  unsigned long long prods = 0;
  const double amax = GATED ? *a.amax : 0.0;
  for (int w = a.w0 + blockIdx.x; w < a.w1; w += gridDim.x) {
    const int row = a.perm[w];
    const int c0 = a.c_rp[row], c1 = a.c_rp[row + 1];
    if (c0 == c1) continue;
    const int a0 = a.a_rp[row], a1 = a.a_rp[row + 1];
    const long long aoff0 = a.a_off[a0], alen = a.a_off[a1] - aoff0;
    const bool staged = alen <= (long long)a.row_cap;
    __syncthreads();  // the previous row's reads of srow and wtab are done
    if (threadIdx.x == 0) {
      s_lo = INT32_MAX;
      s_hi = -1;
    }
    if (staged)
      for (long long e = threadIdx.x; e < alen; e += blockDim.x) srow[e] = A[aoff0 + e];
    __syncthreads();
    int lo = INT32_MAX, hi = -1;
    for (int as = a0 + threadIdx.x; as < a1; as += blockDim.x) {
      const int k = a.a_ci[as];
      lo = min(lo, k);
      hi = max(hi, k);
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, off));
      hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, off));
    }
    if (lane == 0 && hi >= 0) {
      atomicMin(&s_lo, lo);
      atomicMax(&s_hi, hi);
    }
    __syncthreads();
    const int kmin = s_lo;
    const int span = (a1 > a0 && s_hi - kmin < kWinCap) ? s_hi - kmin + 1 : 0;
    for (int t = threadIdx.x; t < span; t += blockDim.x) wtab[t] = -1;
    __syncthreads();
    if (span)
      for (int as = a0 + threadIdx.x; as < a1; as += blockDim.x) wtab[a.a_ci[as] - kmin] = as;
    __syncthreads();
    const double row_eps = gate_eps(GATED ? a.mode : kGateSum, a.thr, amax, a1 - a0, 0);
    // A's values at their offsets in A: the staged copy (generic loads that
    // meet shared memory) or A itself
    const T* Ab = staged ? reinterpret_cast<const T*>(reinterpret_cast<uintptr_t>(srow) -
                                                      static_cast<uintptr_t>(aoff0) * sizeof(T))
                         : A;
    for (int p = c0 + warp; p < c1; p += kNumWarpsCta)
      numeric_block<T, R, GATED>(a, Ab, B, C, p, R, a0, a1, kmin, span, wtab, plist, lane, row_eps, amax, prods);
  }
  if (lane == 0 && prods) atomicAdd(a.products, prods);
}

// FP32 product results into the FP64 values of C.
__global__ void widen_f32_kernel(const float* __restrict__ in, double* __restrict__ out, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = (double)in[i];
}

// The item count is on the device: the grid covers the rows' bound of one
// item per kNumItem C blocks plus one per row, up to 16 CTAs per SM (more
// CTAs than fit at once, so the SMs that finish their items early take new
// CTAs: measured 5 % faster on the McWeeny products than one resident wave).
template <typename T, int R>
static int launch_numeric_r(const NumArgs& x, int64_t max_items, const T* A, const T* B, T* C, cudaStream_t s) {
  const int64_t want = (max_items + kNumWarpsCta - 1) / kNumWarpsCta;
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(want, (int64_t)sm_count() * 16));
  const bool gated = x.mode != kGateSum || x.bound_out || !x.drop;
  // FP64 tensor-core products: a CTA per C row, A's row in shared memory
  // (measured 4.5 % faster on the McWeeny products; FP32 products, on
  // scalar FMAs, ran 6 % slower this way and keep the item kernel)
  if constexpr (std::is_same<T, double>::value && R != 0) {
    if (x.window && x.perm) {
      const NumArgs& xr = x;
      const int rgrid = std::max(1, std::min(x.w1 - x.w0, sm_count() * 16));
      const size_t smem = (size_t)x.row_cap * sizeof(double);
      static bool attr[2][kMaxDevices] = {};
      const int dev = current_device();
      if (!attr[gated][dev]) {
        VBG_CUDA(cudaFuncSetAttribute(gated ? spgemm_numeric_row_kernel<T, R, true>
                                            : spgemm_numeric_row_kernel<T, R, false>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        attr[gated][dev] = true;
      }
      if (gated) {
        spgemm_numeric_row_kernel<T, R, true><<<rgrid, kNumWarpsCta * 32, smem, s>>>(xr, A, B, C);
      } else {
        spgemm_numeric_row_kernel<T, R, false><<<rgrid, kNumWarpsCta * 32, smem, s>>>(xr, A, B, C);
      }
      return 0;
    }
  }
  if constexpr (std::is_same<T, float>::value) {
    if (gated) return fail(VBG_E_ARG, "gated products run in FP64 only");
    spgemm_numeric_kernel<T, R, false><<<grid, kNumWarpsCta * 32, 0, s>>>(x, A, B, C);
  } else if (gated) {
    spgemm_numeric_kernel<T, R, true><<<grid, kNumWarpsCta * 32, 0, s>>>(x, A, B, C);
  } else {
    spgemm_numeric_kernel<T, R, false><<<grid, kNumWarpsCta * 32, 0, s>>>(x, A, B, C);
  }
  return 0;
}

template <typename T>
static int launch_numeric(int r, const NumArgs& x, int64_t max_items, const T* A, const T* B, T* C,
                          cudaStream_t s) {
  switch (r) {
    case 1: return launch_numeric_r<T, 1>(x, max_items, A, B, C, s);
    case 2: return launch_numeric_r<T, 2>(x, max_items, A, B, C, s);
    case 3: return launch_numeric_r<T, 3>(x, max_items, A, B, C, s);
    case 4: return launch_numeric_r<T, 4>(x, max_items, A, B, C, s);
    case 5: return launch_numeric_r<T, 5>(x, max_items, A, B, C, s);
    case 6: return launch_numeric_r<T, 6>(x, max_items, A, B, C, s);
    case 7: return launch_numeric_r<T, 7>(x, max_items, A, B, C, s);
    case 8: return launch_numeric_r<T, 8>(x, max_items, A, B, C, s);
    default: return launch_numeric_r<T, 0>(x, max_items, A, B, C, s);
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
                                int self_cols, int64_t* __restrict__ need) {
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
      if (self_cols) {  // A's own column k joins the row too
        bound += 1;
        lo = min(lo, k);
        hi = max(hi, k);
      }
    }
    if (self_cols && lane == 0) {  // and the diagonal
      bound += 1;
      lo = min(lo, i);
      hi = max(hi, i);
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

// Numeric work items, rows in class order (perm): a row of C with b blocks
// gives ceil(b / kNumItem) items {row, first C slot, C slots}.
__global__ void item_count_kernel(int n, const int* __restrict__ perm, const int* __restrict__ c_rp,
                                  int* __restrict__ cnt) {
  for (int w = blockIdx.x * blockDim.x + threadIdx.x; w < n; w += gridDim.x * blockDim.x) {
    const int row = perm[w];
    cnt[w] = (c_rp[row + 1] - c_rp[row] + kNumItem - 1) / kNumItem;
  }
}

__global__ void item_fill_kernel(int n, const int* __restrict__ perm, const int* __restrict__ c_rp,
                                 const int* __restrict__ start, int4* __restrict__ items) {
  for (int w = blockIdx.x * blockDim.x + threadIdx.x; w < n; w += gridDim.x * blockDim.x) {
    const int row = perm[w];
    const int p0 = c_rp[row], nb = c_rp[row + 1] - p0;
    int f = start[w];
    for (int o = 0; o < nb; o += kNumItem) items[f++] = make_int4(row, p0 + o, min(kNumItem, nb - o), 0);
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

// Which gates a product runs with (kGate*), and what it reads and leaves.
struct GateSpec {
  int mode = kGateSum;
  const double* amax = nullptr;         // gated modes: largest block norm of A (device)
  const double* left_norms = nullptr;   // per A slot (device); default: A's block norms
  const double* right_norms = nullptr;  // per B slot (device); default: B's block norms
  DevBuf* bound_out = nullptr;          // filled with each C slot's kept pair-norm sum
  bool drop = true;                     // drop finished blocks below the threshold
  bool self_cols = false;               // kGatePoly: A's columns and the diagonal join every row
};

// The thresholded product C = A B; with `upper`, only its block columns at
// or above each row (the symbolic phase skips the others, and the numeric
// phase follows C's pattern).
static int spgemm_run(const vbg_matrix* A, const vbg_matrix* B, double thr, int upper, vbg_matrix** Cout,
                      int64_t* stats, cudaStream_t s, int precision = VBG_PREC_F64,
                      const GateSpec& gate = GateSpec{}) {
  VBG_CHECK(A && B && Cout, VBG_E_ARG, "null argument");
  VBG_CHECK(A->dtype == B->dtype, VBG_E_ARG, "A and B must have the same dtype");
  VBG_CHECK(precision == VBG_PREC_F64 || (precision == VBG_PREC_F32 && A->dtype == VBG_F64), VBG_E_ARG,
            "precision must be VBG_PREC_F64, or VBG_PREC_F32 for real matrices");
  VBG_CHECK(A->n == B->n && A->h_bsz == B->h_bsz, VBG_E_ARG, "spmm: A's columns and B's rows differ");
  const int n = A->n;
  int rc;
  // block norms of both operands (cached per call)
  DevBuf nA(s), nB(s), cnt(s), err(s), gtab(s), rows_dev(s);
  const double* normsA = gate.left_norms;
  const double* normsB = gate.right_norms;
  if (!normsA) {
    if ((rc = nA.ensure(std::max<int64_t>(A->nnzb, 1) * 8))) return rc;
    if ((rc = block_norms_dev(A, nA.as<double>(), s))) return rc;
    normsA = nA.as<double>();
  }
  if (!normsB) {
    if ((rc = nB.ensure(std::max<int64_t>(B->nnzb, 1) * 8))) return rc;
    if ((rc = block_norms_dev(B, nB.as<double>(), s))) return rc;
    normsB = nB.as<double>();
  }
  VBG_CHECK(gate.mode == kGateSum || gate.amax, VBG_E_ARG, "gated product without the operand's largest norm");
  VBG_CHECK(!(gate.bound_out && gate.drop), VBG_E_ARG, "pair-norm bounds of a dropped product");
  if ((rc = cnt.ensure((n + 1) * sizeof(int)))) return rc;
  if ((rc = err.ensure(16))) return rc;
  VBG_CUDA(cudaMemsetAsync(err.p, 0, 16, s));
  VBG_CUDA(cudaMemsetAsync(cnt.p, 0, (n + 1) * sizeof(int), s));
  const int serial_b = B->dup_cols ? 1 : 0;

  // symbolic table sizes, computed on the device (sym_need_kernel)
  // page-locked staging of this thread's calls (each use completes before
  // the call returns)
  thread_local HostBuf h_rows;
  std::vector<int64_t> need(n, -1);
  if (n) {
    DevBuf dneed(s);
    if ((rc = dneed.ensure(n * sizeof(int64_t)))) return rc;
    if ((rc = h_rows.ensure(n * sizeof(int64_t)))) return rc;
    const int g = std::max(1, std::min((n + 7) / 8, sm_count() * 16));
    sym_need_kernel<<<g, 256, 0, s>>>(n, A->row_ptr.as<int>(), A->col_ind.as<int>(), B->row_ptr.as<int>(),
                                      B->col_ind.as<int>(), upper, gate.self_cols ? 1 : 0, dneed.as<int64_t>());
    VBG_CUDA(cudaGetLastError());
    VBG_CUDA(cudaMemcpyAsync(h_rows.p, dneed.p, n * sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    VBG_CUDA(cudaStreamSynchronize(s));
    std::memcpy(need.data(), h_rows.p, n * sizeof(int64_t));
  }
  auto sym_bins = make_bins(need);
  SymArgs sa{};
  sa.a_rp = A->row_ptr.as<int>();
  sa.a_ci = A->col_ind.as<int>();
  sa.nA = normsA;
  sa.b_rp = B->row_ptr.as<int>();
  sa.b_ci = B->col_ind.as<int>();
  sa.nB = normsB;
  sa.mode = gate.mode;
  sa.amax = gate.amax;
  sa.self_cols = gate.self_cols ? 1 : 0;
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

  // numeric work items on the device, rows in class order (C has A's rows and
  // their grouping by block size); one launch per class of block sizes <= 8,
  // else one launch over all rows
  const bool small = std::max(A->max_bs, B->max_bs) <= 8;
  const int64_t max_items = cnnzb / kNumItem + n;
  DevBuf items(s), istart(s), icnt(s);
  if ((rc = items.ensure(std::max<int64_t>(max_items, 1) * sizeof(int4)))) return rc;
  if ((rc = istart.ensure((n + 1) * sizeof(int)))) return rc;
  if ((rc = icnt.ensure((n + 1) * sizeof(int)))) return rc;
  VBG_CUDA(cudaMemsetAsync(icnt.p, 0, (n + 1) * sizeof(int), s));
  if (n) {
    const int g = std::max(1, std::min((n + 255) / 256, sm_count() * 8));
    item_count_kernel<<<g, 256, 0, s>>>(n, C->row_perm.as<int>(), C->row_ptr.as<int>(), icnt.as<int>());
    VBG_CUDA(cudaGetLastError());
  }
  if ((rc = exclusive_sum_int(icnt.as<int>(), istart.as<int>(), n + 1, s))) return rc;
  if (n) {
    const int g = std::max(1, std::min((n + 255) / 256, sm_count() * 8));
    item_fill_kernel<<<g, 256, 0, s>>>(n, C->row_perm.as<int>(), C->row_ptr.as<int>(), istart.as<int>(),
                                       items.as<int4>());
    VBG_CUDA(cudaGetLastError());
  }
  struct Launch {
    int r, w0, w1;
  };
  std::vector<Launch> launches;
  if (small) {
    for (const auto& seg : C->class_segs) launches.push_back({seg.r, seg.w0, seg.w1});
  } else if (n) {
    launches.push_back({0, 0, n});
  }
  if ((rc = build_csc_dev(B, s))) return rc;
  NumArgs na{};
  na.a_rp = A->row_ptr.as<int>();
  na.a_ci = A->col_ind.as<int>();
  na.a_off = A->blk_off.as<int64_t>();
  na.nA = normsA;
  na.bt_ptr = B->csc_ptr.as<int>();
  na.bt_row = B->csc_row.as<int>();
  na.bt_slot = B->csc_slot.as<int>();
  na.b_off = B->blk_off.as<int64_t>();
  na.nB = normsB;
  na.mode = gate.mode;
  na.amax = gate.amax;
  na.b_rp = B->row_ptr.as<int>();
  na.drop = gate.drop ? 1 : 0;
  if (gate.bound_out) {
    if ((rc = gate.bound_out->ensure(std::max<int64_t>(cnnzb, 1) * sizeof(double)))) return rc;
    na.bound_out = gate.bound_out->as<double>();
  }
  na.bsz = A->bsz.as<int>();
  na.c_ci = C->col_ind.as<int>();
  na.c_off = C->blk_off.as<int64_t>();
  na.thr = thr;
  na.dup = B->dup_cols ? 1 : 0;
  na.window = (A->dup_cols || B->dup_cols) ? 0 : 1;
  na.perm = C->row_perm.as<int>();
  na.c_rp = C->row_ptr.as<int>();
  na.row_cap = kRowStageCap;
  na.keep = keep.as<unsigned char>();
  na.products = prods.as<unsigned long long>();
  {
    DevBuf c32(s);
    const bool f32 = precision == VBG_PREC_F32;
    if (f32) {
      // FP32 operands (the shadows) and FP32 accumulation; the block norms,
      // the skip and keep rules stay FP64
      if ((rc = ensure_vals32(A, s))) return rc;
      if ((rc = ensure_vals32(B, s))) return rc;
      if ((rc = c32.ensure(std::max<int64_t>(C->nnz, 1) * sizeof(float)))) return rc;
    }
    for (const Launch& L : launches) {
      NumArgs x = na;
      x.items = items.as<int4>();
      x.item_start = istart.as<int>();
      x.w0 = L.w0;
      x.w1 = L.w1;
      // items of these rows: at most one per kNumItem C blocks plus one per row
      const int64_t bound = std::min<int64_t>(max_items, cnnzb / kNumItem + (L.w1 - L.w0));
      if (C->dtype == VBG_C128)
        rc = launch_numeric<cplx>(L.r, x, bound, A->vals.as<cplx>(), B->vals.as<cplx>(), C->vals.as<cplx>(), s);
      else if (f32)
        rc = launch_numeric<float>(L.r, x, bound, A->vals32.as<float>(), B->vals32.as<float>(), c32.as<float>(), s);
      else
        rc = launch_numeric<double>(L.r, x, bound, A->vals.as<double>(), B->vals.as<double>(), C->vals.as<double>(),
                                    s);
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
  const int64_t sym_blocks = cnnzb;
  if (gate.drop && thr > 0.0 && (rc = compact_by_mask_dev(C.get(), keep.as<unsigned char>(), s))) return rc;
  if (stats) {
    // the pair count is read back only for the statistics
    unsigned long long hprods = 0;
    VBG_CUDA(cudaMemcpyAsync(&hprods, prods.p, 8, cudaMemcpyDeviceToHost, s));
    VBG_CUDA(cudaStreamSynchronize(s));
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

// ------------------------------------------------ fused triple products
// The reference's square_polynomial_upper, rarh_upper and rhar_upper
// (block_csr.hpp:1803-1853; ops/spmm/square_polynomial.hpp, rarh.hpp,
// rhar.hpp) hold one row of the intermediate per thread and apply the drop
// threshold once, to the finished blocks, with per-row pair gates in
// between.  Here the intermediate is materialised in device memory instead
// (HBM holds it easily at the sizes one GPU takes) and the same gates decide
// which pairs reach it: stage one keeps every column a passing pair reaches
// and records each block's sum of pair norms, stage two gates on those sums,
// and only the final product is dropped below the threshold.  The product
// kernels are the SpGEMM's (gate modes kGateStage1/2, kGatePoly).
namespace vbg {

// out[0] = the largest of v[0, n) (0 for n == 0); one CTA.
__global__ void max_value_kernel(const double* __restrict__ v, int64_t n, double* out) {
  __shared__ double red[32];
  double m = 0.0;
  for (int64_t i = threadIdx.x; i < n; i += blockDim.x) m = fmax(m, v[i]);
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, off));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) m = fmax(m, red[w]);
    out[0] = fmax(m, red[0]);
  }
}

__device__ __forceinline__ double cmul_re(double ar, double ai, double br, double bi) { return ar * br - ai * bi; }
__device__ __forceinline__ double cmul_im(double ar, double ai, double br, double bi) { return ar * bi + ai * br; }

// C = c2 S + c1 A + c0 I on S's pattern (which holds A's upper columns and
// the diagonal), in the reference's order: every block scaled by c2, then
// c1 A_ij added for each of A's blocks (i, j), then c0 on the diagonal; the
// keep flag of each finished block (norm >= threshold, all for thr <= 0).
// A warp per block row, lanes over a block's elements.
template <typename T>
__global__ void poly_epilogue_kernel(int n, const int* __restrict__ c_rp, const int* __restrict__ c_ci,
                                     const int64_t* __restrict__ c_off, T* __restrict__ cv,
                                     const int* __restrict__ a_rp, const int* __restrict__ a_ci,
                                     const int64_t* __restrict__ a_off, const T* __restrict__ av,
                                     const int* __restrict__ bsz, cplx c2, cplx c1, cplx c0, double thr,
                                     unsigned char* __restrict__ keep) {
  const int lane = threadIdx.x & 31;
  const int warps = gridDim.x * (blockDim.x >> 5);
  for (int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); i < n; i += warps) {
    const int r = bsz[i];
    const int a0 = a_rp[i], a1 = a_rp[i + 1];
    for (int p = c_rp[i]; p < c_rp[i + 1]; ++p) {
      const int j = c_ci[p];
      const int c = bsz[j];
      // A's slots of column j in row i (columns ascending; duplicates each add)
      int lo = a0, hi = a1;
      while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (a_ci[mid] < j) lo = mid + 1;
        else hi = mid;
      }
      T* blk = cv + c_off[p];
      double sq = 0.0;
      for (int e = lane; e < r * c; e += 32) {
        double vr, vi = 0.0;
        if constexpr (sizeof(T) == sizeof(cplx)) {
          const cplx x = reinterpret_cast<const cplx*>(blk)[e];
          vr = cmul_re(x.re, x.im, c2.re, c2.im);
          vi = cmul_im(x.re, x.im, c2.re, c2.im);
          for (int s = lo; s < a1 && a_ci[s] == j; ++s) {
            const cplx y = reinterpret_cast<const cplx*>(av + a_off[s])[e];
            vr += cmul_re(c1.re, c1.im, y.re, y.im);
            vi += cmul_im(c1.re, c1.im, y.re, y.im);
          }
          if (i == j && e % (r + 1) == 0) {
            vr += c0.re;
            vi += c0.im;
          }
          reinterpret_cast<cplx*>(blk)[e] = cplx{vr, vi};
        } else {
          vr = reinterpret_cast<const double*>(blk)[e] * c2.re;
          for (int s = lo; s < a1 && a_ci[s] == j; ++s) vr += c1.re * reinterpret_cast<const double*>(av + a_off[s])[e];
          if (i == j && e % (r + 1) == 0) vr += c0.re;
          reinterpret_cast<double*>(blk)[e] = vr;
        }
        sq += vr * vr + vi * vi;
      }
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) sq += __shfl_xor_sync(0xffffffffu, sq, off);
      if (lane == 0) keep[p] = (thr <= 0.0 || sqrt(sq) >= thr) ? 1 : 0;
    }
  }
}

// Block norms of m and their largest value, on the device.
static int norms_and_max(const vbg_matrix* m, DevBuf& norms, DevBuf& mx, cudaStream_t s) {
  int rc;
  if ((rc = norms.ensure(std::max<int64_t>(m->nnzb, 1) * 8))) return rc;
  if ((rc = mx.ensure(8))) return rc;
  if ((rc = block_norms_dev(m, norms.as<double>(), s))) return rc;
  max_value_kernel<<<1, 1024, 0, s>>>(norms.as<double>(), m->nnzb, mx.as<double>());
  VBG_CUDA(cudaGetLastError());
  return 0;
}

// A B A^H (rhar = false; A and B Hermitian) or A^H B A (rhar = true; B
// Hermitian), upper block triangle.
static int fused_triple(const vbg_matrix* A, const vbg_matrix* B, double thr, bool rhar, vbg_matrix** out,
                        cudaStream_t s) {
  VBG_CHECK(A && B && out, VBG_E_ARG, "null argument");
  VBG_CHECK(A->dtype == B->dtype, VBG_E_ARG, "A and B must have the same dtype");
  VBG_CHECK(A->n == B->n && A->h_bsz == B->h_bsz, VBG_E_ARG, "A and B must share the block structure's sizes");
  int rc;
  DevBuf nA(s), amax(s), nL(s), lmax(s), bound(s);
  if ((rc = norms_and_max(A, nA, amax, s))) return rc;
  const vbg_matrix* L = A;
  std::unique_ptr<vbg_matrix> Ah;
  if (rhar) {
    // the left factors of row i are A's column i, conjugate-transposed
    vbg_matrix* t = nullptr;
    if ((rc = vbg_matrix_transpose(A, &t, s))) return rc;
    Ah.reset(t);
    L = t;
    if ((rc = norms_and_max(t, nL, lmax, s))) return rc;
  }
  GateSpec g1;
  g1.mode = kGateStage1;
  g1.amax = amax.as<double>();
  g1.left_norms = rhar ? nL.as<double>() : nA.as<double>();
  g1.bound_out = &bound;
  g1.drop = false;
  vbg_matrix* T = nullptr;
  if ((rc = spgemm_run(L, B, thr, 0, &T, nullptr, s, VBG_PREC_F64, g1))) return rc;
  std::unique_ptr<vbg_matrix> Tkeep(T);
  // C[i, j >= i] = sum_l T_il A_lj (A^H's row l is A's row l for rarh)
  GateSpec g2;
  g2.mode = kGateStage2;
  g2.amax = amax.as<double>();
  g2.left_norms = bound.as<double>();
  g2.right_norms = nA.as<double>();
  g2.drop = true;
  return spgemm_run(T, A, thr, 1, out, nullptr, s, VBG_PREC_F64, g2);
}

}  // namespace vbg

extern "C" int vbg_square_polynomial_upper(const vbg_matrix* A, double c2_re, double c2_im, double c1_re,
                                           double c1_im, double c0_re, double c0_im, double threshold,
                                           vbg_matrix** out, void* stream) {
  VBG_CHECK(A && out, VBG_E_ARG, "null argument");
  cudaStream_t s = as_stream(stream);
  int rc;
  DevBuf nA(s), amax(s), keep(s);
  if ((rc = norms_and_max(A, nA, amax, s))) return rc;
  GateSpec g;
  g.mode = kGatePoly;
  g.amax = amax.as<double>();
  g.left_norms = nA.as<double>();
  g.right_norms = nA.as<double>();
  g.drop = false;
  g.self_cols = true;
  vbg_matrix* S = nullptr;
  if ((rc = spgemm_run(A, A, threshold, 1, &S, nullptr, s, VBG_PREC_F64, g))) return rc;
  std::unique_ptr<vbg_matrix> C(S);
  if (C->nnzb) {
    if ((rc = keep.ensure(C->nnzb))) return rc;
    const int grid = std::max(1, std::min((C->n + 7) / 8, sm_count() * 8));
    const cplx c2{c2_re, c2_im}, c1{c1_re, c1_im}, c0{c0_re, c0_im};
    if (C->dtype == VBG_C128)
      poly_epilogue_kernel<cplx><<<grid, 256, 0, s>>>(C->n, C->row_ptr.as<int>(), C->col_ind.as<int>(),
                                                      C->blk_off.as<int64_t>(), C->vals.as<cplx>(),
                                                      A->row_ptr.as<int>(), A->col_ind.as<int>(),
                                                      A->blk_off.as<int64_t>(), A->vals.as<cplx>(),
                                                      A->bsz.as<int>(), c2, c1, c0, threshold,
                                                      keep.as<unsigned char>());
    else
      poly_epilogue_kernel<double><<<grid, 256, 0, s>>>(C->n, C->row_ptr.as<int>(), C->col_ind.as<int>(),
                                                        C->blk_off.as<int64_t>(), C->vals.as<double>(),
                                                        A->row_ptr.as<int>(), A->col_ind.as<int>(),
                                                        A->blk_off.as<int64_t>(), A->vals.as<double>(),
                                                        A->bsz.as<int>(), c2, c1, c0, threshold,
                                                        keep.as<unsigned char>());
    VBG_CUDA(cudaGetLastError());
    if (threshold > 0.0 && (rc = compact_by_mask_dev(C.get(), keep.as<unsigned char>(), s))) return rc;
  }
  *out = C.release();
  return 0;
}

extern "C" int vbg_rarh_upper(const vbg_matrix* A, const vbg_matrix* B, double threshold, vbg_matrix** out,
                              void* stream) {
  return fused_triple(A, B, threshold, false, out, as_stream(stream));
}

extern "C" int vbg_rhar_upper(const vbg_matrix* A, const vbg_matrix* B, double threshold, vbg_matrix** out,
                              void* stream) {
  return fused_triple(A, B, threshold, true, out, as_stream(stream));
}

extern "C" int vbg_matrix_complete_hermitian(vbg_matrix* m, void* stream) {
  VBG_CHECK(m, VBG_E_ARG, "null matrix");
  return complete_hermitian_dev(m, as_stream(stream));
}
