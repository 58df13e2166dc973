// Sparse apply kernels: y = A x, Y = A X, their adjoints, the fused Chebyshev
// step (recurrence update + moment dot products in one pass) and the KPM
// moment loop built on it.
//
// Reference behaviour replaced:
//   BlockSpMat::mult / mult_dense / mult_adjoint / mult_dense_adjoint
//     vbcsr/core/block_csr.hpp:985-1050
//   row-direct apply  vbcsr/core/detail/kernels/vbcsr_apply.hpp:193-244 (mult),
//     :277-340 (mult_dense), :342-424 (adjoint)
//   per-block kernels rm_gemv / rm_gemm
//     vbcsr/core/detail/kernels/rowmajor_kernels.hpp:45-185,552-600
//   Chebyshev loop bodies examples/ex08_graphene_dos.py:99-114,
//     examples/inp_nanocrystal_dos/kpm.py:40-74, vbcsr/utils.py:71-126
//
// Layout: one warp per output block row.  For a plain vector the 32 lanes are
// split into (block, row-within-block) pairs, each lane reducing one r x c
// block row against its x strip; for a multivector the lanes cover the padded
// row of X (16-byte vectors per lane: 2 FP64, 4 FP32 or 1 complex) and lane
// groups split the row's blocks when the row is narrower than a warp.  Rows
// are visited in block-size-class order and the block size r is a
// compile-time constant inside each class body.
#include <algorithm>
#include <atomic>
#include <cstring>
#include <mutex>
#include <type_traits>

#include "vbg_internal.cuh"

namespace vbg {

constexpr int kWarps = 8;
constexpr int kThreads = kWarps * 32;

struct ApplyArgs {
  int n_rows;                // output block rows
  const int* order;          // visiting order of output rows (nullptr = natural)
  const int* ptr;            // entry range per output row (row_ptr or csc_ptr)
  const int* ent_slot;       // adjoint: slot of each entry (forward: entry == slot)
  const int* ent_src;        // source block of each entry (col_ind or csc_row)
  const int* bsz;
  const int64_t* scal_off;
  const int64_t* blk_off;
  const int2* slot_meta;     // forward: per slot {first X row of the block column, rows << 8 | cols}
  const int64_t* koff;       // pipelined kernel: per-slot offsets of the kernel-layout values
  const int4* spans;         // pipelined kernel: spans, FP32 layout offsets, each block row's span range
  const int64_t* span_koff32;
  const int* row_sptr;
  int ld;                    // leading dimension of X/Y in elements (1 = vector)
  // epilogue  Y = alpha * (A X) + beta * X + gamma * Xprev
  double alpha, beta, gamma;
  const void* X;
  const void* Xprev;
  void* Y;
  const void* dotw;          // dot partner for dots[0] (nullptr -> X)
  void* acc;                 // acc += acc_coef * Y (nullptr -> none)
  double cre, cim;
  int want_dots;
  double* row_dots;          // with want_dots: per block row (d0, d1) here instead of the grid reduction
  double* partials;
  unsigned* counter;
  double* dots_out;
  int max_ctas;              // CTAs `partials` has room for (0: max_total_ctas())
  // vector apply: ranges each CTA prefetches its share of into L2 at start
  // (16-byte aligned; set when the whole working set fits L2)
  int npf;
  const void* pf_ptr[4];
  long long pf_bytes[4];
  // scalar-row vector apply: per scalar row {first slot, count << 8 | row in block}, scalar rows
  const int2* srow;
  int64_t n_scal;
};

template <typename T> struct VT;
template <> struct VT<double> { using raw = double2; static constexpr int E = 2; };
template <> struct VT<float> { using raw = float4; static constexpr int E = 4; };
template <> struct VT<cplx> { using raw = double2; static constexpr int E = 1; };

template <typename T>
struct Vec {
  T v[VT<T>::E];
};

template <typename T>
__device__ __forceinline__ Vec<T> load_vec(const T* base, int64_t vidx) {
  typename VT<T>::raw r = reinterpret_cast<const typename VT<T>::raw*>(base)[vidx];
  Vec<T> out;
  memcpy(&out, &r, sizeof(r));
  return out;
}
template <typename T>
__device__ __forceinline__ void store_vec(T* base, int64_t vidx, const Vec<T>& v) {
  typename VT<T>::raw r;
  memcpy(&r, &v, sizeof(r));
  reinterpret_cast<typename VT<T>::raw*>(base)[vidx] = r;
}

__device__ __forceinline__ double shfl_xor_s(double v, int off) { return __shfl_xor_sync(0xffffffffu, v, off); }
__device__ __forceinline__ float shfl_xor_s(float v, int off) { return __shfl_xor_sync(0xffffffffu, v, off); }
__device__ __forceinline__ cplx shfl_xor_s(cplx v, int off) {
  return {__shfl_xor_sync(0xffffffffu, v.re, off), __shfl_xor_sync(0xffffffffu, v.im, off)};
}
__device__ __forceinline__ double add_s(double a, double b) { return a + b; }
__device__ __forceinline__ float add_s(float a, float b) { return a + b; }
__device__ __forceinline__ cplx add_s(cplx a, cplx b) { return {a.re + b.re, a.im + b.im}; }

// Epilogue for one output element.
template <typename T>
__device__ __forceinline__ T epi_value(const ApplyArgs& a, T sum, int64_t gi) {
  T y = scal_r(a.alpha, sum);
  if (a.beta != 0.0) y = axpy_r(a.beta, static_cast<const T*>(a.X)[gi], y);
  if (a.gamma != 0.0) y = axpy_r(a.gamma, static_cast<const T*>(a.Xprev)[gi], y);
  return y;
}

template <typename T>
__device__ __forceinline__ void epi_finish(const ApplyArgs& a, T y, int64_t gi, double& d0, double& d1) {
  if (a.want_dots) {
    const T xd = a.dotw ? static_cast<const T*>(a.dotw)[gi] : static_cast<const T*>(a.X)[gi];
    d0 += re_dot(xd, y);
    d1 += re_dot(y, y);
  }
  if (a.acc) {
    T* ac = static_cast<T*>(a.acc);
    ac[gi] = cmad(a.cre, a.cim, y, ac[gi]);
  }
}

// ------------------------------------------------------------ vector rows
// Sums the G = 32 / R lane groups' partial rows of one block row and runs the
// epilogue on its R outputs.
template <typename T, int R>
__device__ __forceinline__ void vec_row_finish(const ApplyArgs& a, int row, int lane, T acc, T* wred, double& d0,
                                               double& d1) {
  constexpr int G = 32 / R;
  wred[lane] = acc;
  __syncwarp();
  if (lane < R) {
    T sum = wred[lane];
#pragma unroll
    for (int b = 1; b < G; ++b) sum = add_s(sum, wred[lane + b * R]);
    const int64_t gi = a.scal_off[row] + lane;
    const T y = epi_value(a, sum, gi);
    static_cast<T*>(a.Y)[gi] = y;
    epi_finish(a, y, gi, d0, d1);
  }
  __syncwarp();
}

// Lane l handles block (l / R) of each chunk of G = 32 / R blocks and the
// block row (l % R) inside it.
template <typename T, int R, bool ADJ>
__device__ __forceinline__ void vec_row(const ApplyArgs& a, const T* __restrict__ vals, int row, int lane,
                                        T* wred, double& d0, double& d1) {
  constexpr int G = 32 / R;
  const int bl = lane / R;
  const int o = lane - bl * R;
  const int e0 = a.ptr[row], e1 = a.ptr[row + 1];
  const T* __restrict__ x = static_cast<const T*>(a.X);
  T acc = zero_s<T>();
  if (bl < G) {
    for (int e = e0 + bl; e < e1; e += G) {
      const int src = a.ent_src[e];
      const int s = ADJ ? a.ent_slot[e] : e;
      const int inner = a.bsz[src];
      const T* xp = x + a.scal_off[src];
      const T* ap = vals + a.blk_off[s] + (ADJ ? o : o * inner);
#pragma unroll 4
      for (int q = 0; q < inner; ++q) {
        T av = ap[ADJ ? q * R : q];
        if (ADJ) av = conj_s(av);
        acc = fma_s(av, xp[q], acc);
      }
    }
  }
  vec_row_finish<T, R>(a, row, lane, acc, wred, d0, d1);
}

// Rows wider than 8: lane handles output rows o0 + lane over all entries.
template <typename T, bool ADJ>
__device__ void vec_row_wide(const ApplyArgs& a, const T* __restrict__ vals, int row, int lane, double& d0,
                             double& d1) {
  const int r = a.bsz[row];
  const int e0 = a.ptr[row], e1 = a.ptr[row + 1];
  const T* __restrict__ x = static_cast<const T*>(a.X);
  for (int o0 = 0; o0 < r; o0 += 32) {
    const int o = o0 + lane;
    if (o < r) {
      T acc = zero_s<T>();
      for (int e = e0; e < e1; ++e) {
        const int src = a.ent_src[e];
        const int s = ADJ ? a.ent_slot[e] : e;
        const int inner = a.bsz[src];
        const T* xp = x + a.scal_off[src];
        const T* ap = vals + a.blk_off[s] + (ADJ ? o : (int64_t)o * inner);
        for (int q = 0; q < inner; ++q) {
          T av = ap[ADJ ? (int64_t)q * r : q];
          if (ADJ) av = conj_s(av);
          acc = fma_s(av, xp[q], acc);
        }
      }
      const int64_t gi = a.scal_off[row] + o;
      const T y = epi_value(a, acc, gi);
      static_cast<T*>(a.Y)[gi] = y;
      epi_finish(a, y, gi, d0, d1);
    }
  }
}

// Forward vector rows from the per-slot records: lane j of the warp loads
// slot j's {first X row, shape} and value offset for up to 32 of the row's
// blocks at once, so a block costs one level of dependent loads instead of
// three (column index, then the column's offset and size, then values and X).
// The blocks are then handed out by shuffles, G = 32 / R at a time, lane l
// taking block (l / R) and its row (l % R); the value and X loads of two such
// rounds are issued before their multiply-adds.  The records hold 32-bit X
// offsets and 8-bit block sizes, so the caller takes this path for N < 2^31
// and blocks of at most 255 only.  CH columns of a block row are loaded
// before their multiply-adds (fewer for complex values, whose staging
// registers would otherwise set the kernel's occupancy).
template <typename T, int R, int CH = 8>
__device__ __forceinline__ void vec_row_meta(const ApplyArgs& a, const T* __restrict__ vals, int row, int lane,
                                             T* wred, double& d0, double& d1) {
  constexpr int G = 32 / R;
  const int bl = lane / R;
  const int o = lane - bl * R;
  const int e0 = a.ptr[row], e1 = a.ptr[row + 1];
  const T* __restrict__ x = static_cast<const T*>(a.X);
  T acc = zero_s<T>();
  for (int base = e0; base < e1; base += 32) {
    const int cnt = min(32, e1 - base);
    int xo = 0, cs = 0;
    long long vo = 0;
    if (lane < cnt) {
      const int2 mt = __ldg(a.slot_meta + base + lane);
      xo = mt.x;
      cs = mt.y & 0xff;
      vo = __ldg(a.blk_off + base + lane);
    }
    for (int j0 = 0; j0 < cnt; j0 += G) {
      const int j = j0 + bl;
      const int jx = __shfl_sync(0xffffffffu, xo, j & 31);
      const int jc = __shfl_sync(0xffffffffu, cs, j & 31);
      const long long jv = __shfl_sync(0xffffffffu, vo, j & 31);
      if (bl < G && j < cnt) {
        const T* __restrict__ ap = vals + jv + (long long)o * jc;
        const T* __restrict__ xp = x + (unsigned)jx;
        for (int q0 = 0; q0 < jc; q0 += CH) {  // block columns wider than CH take several rounds
          T av[CH], xv[CH];
#pragma unroll
          for (int q = 0; q < CH; ++q) {
            av[q] = q0 + q < jc ? ap[q0 + q] : zero_s<T>();
            xv[q] = q0 + q < jc ? xp[q0 + q] : zero_s<T>();
          }
#pragma unroll
          for (int q = 0; q < CH; ++q) acc = fma_s(av[q], xv[q], acc);
        }
      }
    }
  }
  vec_row_finish<T, R>(a, row, lane, acc, wred, d0, d1);
}

template <typename T, int CH = 8>
__device__ __forceinline__ bool dispatch_vec_row_meta(const ApplyArgs& a, const T* __restrict__ vals, int row,
                                                      int lane, T* wred, double& d0, double& d1) {
  switch (a.bsz[row]) {
    case 1: vec_row_meta<T, 1, CH>(a, vals, row, lane, wred, d0, d1); return true;
    case 2: vec_row_meta<T, 2, CH>(a, vals, row, lane, wred, d0, d1); return true;
    case 3: vec_row_meta<T, 3, CH>(a, vals, row, lane, wred, d0, d1); return true;
    case 4: vec_row_meta<T, 4, CH>(a, vals, row, lane, wred, d0, d1); return true;
    case 5: vec_row_meta<T, 5, CH>(a, vals, row, lane, wred, d0, d1); return true;
    case 6: vec_row_meta<T, 6, CH>(a, vals, row, lane, wred, d0, d1); return true;
    case 7: vec_row_meta<T, 7, CH>(a, vals, row, lane, wred, d0, d1); return true;
    case 8: vec_row_meta<T, 8, CH>(a, vals, row, lane, wred, d0, d1); return true;
    default: return false;
  }
}

// ------------------------------------------------------- multivector rows
// lanes [grp*LPR, grp*LPR + LPR) cover 16-byte vectors of the padded X row;
// the G lane groups take every G-th block of the row and are summed by
// butterfly shuffles at the end.  RM output rows per pass (R <= 8 exact).
template <typename T, int RM, bool ADJ>
__device__ __forceinline__ void mv_rows(const ApplyArgs& a, const T* __restrict__ vals, int row, int lane, int lpr,
                                        int G, int o0, int rcount, int rfull, double& d0, double& d1) {
  constexpr int E = VT<T>::E;
  const int grp = lane / lpr;
  const int vl = lane - grp * lpr;
  const int nvec = a.ld / E;
  const int e0 = a.ptr[row], e1 = a.ptr[row + 1];
  const T* __restrict__ X = static_cast<const T*>(a.X);
  for (int v0 = 0; v0 < nvec; v0 += lpr) {
    const int vi = v0 + vl;
    const bool valid = grp < G && vi < nvec;
    Vec<T> acc[RM];
#pragma unroll
    for (int o = 0; o < RM; ++o)
#pragma unroll
      for (int u = 0; u < E; ++u) acc[o].v[u] = zero_s<T>();
    if (valid) {
      for (int e = e0 + grp; e < e1; e += G) {
        const int src = a.ent_src[e];
        const int s = ADJ ? a.ent_slot[e] : e;
        const int inner = a.bsz[src];
        const int64_t xrow0 = a.scal_off[src];
        const T* ab = vals + a.blk_off[s];
        for (int q = 0; q < inner; ++q) {
          const Vec<T> xv = load_vec(X, (xrow0 + q) * nvec + vi);
#pragma unroll
          for (int o = 0; o < RM; ++o) {
            if (o < rcount) {
              T av = ADJ ? ab[(int64_t)q * rfull + o0 + o] : ab[(int64_t)(o0 + o) * inner + q];
              if (ADJ) av = conj_s(av);
#pragma unroll
              for (int u = 0; u < E; ++u) acc[o].v[u] = fma_s(av, xv.v[u], acc[o].v[u]);
            }
          }
        }
      }
    }
    if (G > 1) {
      for (int off = lpr; off < G * lpr; off <<= 1) {
#pragma unroll
        for (int o = 0; o < RM; ++o)
#pragma unroll
          for (int u = 0; u < E; ++u) acc[o].v[u] = add_s(acc[o].v[u], shfl_xor_s(acc[o].v[u], off));
      }
    }
    if (grp == 0 && vi < nvec) {
#pragma unroll
      for (int o = 0; o < RM; ++o) {
        if (o < rcount) {
          const int64_t grow = a.scal_off[row] + o0 + o;
          const int64_t vidx = grow * nvec + vi;
          Vec<T> y;
          if (a.beta == 0.0 && a.gamma == 0.0 && !a.want_dots && !a.acc) {
#pragma unroll
            for (int u = 0; u < E; ++u) y.v[u] = scal_r(a.alpha, acc[o].v[u]);
          } else {
            Vec<T> xs, xp, xd, ac;
            if (a.beta != 0.0 || (a.want_dots && !a.dotw)) xs = load_vec(X, vidx);
            if (a.gamma != 0.0) xp = load_vec(static_cast<const T*>(a.Xprev), vidx);
            if (a.want_dots) xd = a.dotw ? load_vec(static_cast<const T*>(a.dotw), vidx) : xs;
            if (a.acc) ac = load_vec(static_cast<const T*>(a.acc), vidx);
#pragma unroll
            for (int u = 0; u < E; ++u) {
              T yy = scal_r(a.alpha, acc[o].v[u]);
              if (a.beta != 0.0) yy = axpy_r(a.beta, xs.v[u], yy);
              if (a.gamma != 0.0) yy = axpy_r(a.gamma, xp.v[u], yy);
              y.v[u] = yy;
              if (a.want_dots) {
                d0 += re_dot(xd.v[u], yy);
                d1 += re_dot(yy, yy);
              }
              if (a.acc) ac.v[u] = cmad(a.cre, a.cim, yy, ac.v[u]);
            }
            if (a.acc) store_vec(static_cast<T*>(a.acc), vidx, ac);
          }
          store_vec(static_cast<T*>(a.Y), vidx, y);
        }
      }
    }
  }
}

template <typename T, bool ADJ>
__device__ __forceinline__ void dispatch_vec_row(const ApplyArgs& a, const T* __restrict__ vals, int row, int lane,
                                                 T* wred, double& d0, double& d1) {
  switch (a.bsz[row]) {
    case 1: vec_row<T, 1, ADJ>(a, vals, row, lane, wred, d0, d1); break;
    case 2: vec_row<T, 2, ADJ>(a, vals, row, lane, wred, d0, d1); break;
    case 3: vec_row<T, 3, ADJ>(a, vals, row, lane, wred, d0, d1); break;
    case 4: vec_row<T, 4, ADJ>(a, vals, row, lane, wred, d0, d1); break;
    case 5: vec_row<T, 5, ADJ>(a, vals, row, lane, wred, d0, d1); break;
    case 6: vec_row<T, 6, ADJ>(a, vals, row, lane, wred, d0, d1); break;
    case 7: vec_row<T, 7, ADJ>(a, vals, row, lane, wred, d0, d1); break;
    case 8: vec_row<T, 8, ADJ>(a, vals, row, lane, wred, d0, d1); break;
    default: vec_row_wide<T, ADJ>(a, vals, row, lane, d0, d1); break;
  }
}

// Fixed-order two-value reduction across the grid: per-CTA partials, then
// the last CTA to finish sums them in a fixed tree and resets the counter.
// Blocks have at most 1024 threads.
__device__ void grid_reduce2(double d0, double d1, double* partials, unsigned* counter, double* out, int part_base,
                             int total) {
  __shared__ double red[32][2];
  __shared__ bool is_last;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    d0 += __shfl_xor_sync(0xffffffffu, d0, off);
    d1 += __shfl_xor_sync(0xffffffffu, d1, off);
  }
  if (lane == 0) {
    red[warp][0] = d0;
    red[warp][1] = d1;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double s0 = 0.0, s1 = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
      s0 += red[w][0];
      s1 += red[w][1];
    }
    partials[2 * (part_base + blockIdx.x)] = s0;
    partials[2 * (part_base + blockIdx.x) + 1] = s1;
    __threadfence();
    const unsigned prev = atomicAdd(counter, 1u);
    is_last = (prev == (unsigned)total - 1);
  }
  __syncthreads();
  if (!is_last) return;
  __threadfence();
  double s0 = 0.0, s1 = 0.0;
  for (int b = threadIdx.x; b < total; b += blockDim.x) {
    s0 += __ldcg(partials + 2 * b);
    s1 += __ldcg(partials + 2 * b + 1);
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    s0 += __shfl_xor_sync(0xffffffffu, s0, off);
    s1 += __shfl_xor_sync(0xffffffffu, s1, off);
  }
  __syncthreads();
  if (lane == 0) {
    red[warp][0] = s0;
    red[warp][1] = s1;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double t0 = 0.0, t1 = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
      t0 += red[w][0];
      t1 += red[w][1];
    }
    out[0] = t0;
    out[1] = t1;
    *counter = 0u;
  }
}

// Per-row dot output (batched recurrences): sums this row's lane partials
// over the warp and writes them; the caller's accumulators are untouched.
__device__ __forceinline__ void write_row_dots(double* row_dots, int row, double r0, double r1) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    r0 += __shfl_xor_sync(0xffffffffu, r0, off);
    r1 += __shfl_xor_sync(0xffffffffu, r1, off);
  }
  if ((threadIdx.x & 31) == 0) {
    row_dots[2 * row] = r0;
    row_dots[2 * row + 1] = r1;
  }
}

// This CTA's share of [p, p + bytes) prefetched into L2 by bulk prefetches
// (16-byte units, 64 KiB per instruction; a tail under 16 bytes is left to
// the loads).  p is 16-byte aligned.
__device__ __forceinline__ void prefetch_share_l2(const void* p, long long bytes) {
  const long long units = bytes >> 4;
  const long long per = (units + gridDim.x - 1) / gridDim.x;
  long long u = per * blockIdx.x;
  const long long u1 = min(units, u + per);
  const char* c = static_cast<const char*>(p);
  for (; u < u1; u += 4096) {
    const unsigned n = static_cast<unsigned>(min(u1 - u, 4096ll) << 4);
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;\n" ::"l"(c + (u << 4)), "r"(n) : "memory");
  }
}

// Plain vectors: one launch over all rows, block size dispatched per warp.
// For a working set that fits L2 every CTA first asks L2 for its share of
// the values, the slot records and X, so the warps' dependent loads (row
// range, then records, then values and X) meet L2 instead of HBM latency.
template <typename T, bool ADJ>
__global__ void __launch_bounds__(kThreads) apply_vec_kernel(ApplyArgs a, const T* __restrict__ vals, int part_base,
                                                             int total) {
  __shared__ T wred_all[kThreads];
  if (a.npf && threadIdx.x == 0)
    for (int r = 0; r < a.npf; ++r) prefetch_share_l2(a.pf_ptr[r], a.pf_bytes[r]);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  T* wred = wred_all + warp * 32;
  double d0 = 0.0, d1 = 0.0;
  for (int w = blockIdx.x * kWarps + warp; w < a.n_rows; w += gridDim.x * kWarps) {
    // with the slot records, rows in their own order (one warp per row:
    // grouping by size buys nothing here and costs a dependent load)
    const bool meta = !ADJ && a.slot_meta;
    if (meta && dispatch_vec_row_meta<T>(a, vals, w, lane, wred, d0, d1)) continue;
    const int row = (meta || !a.order) ? w : a.order[w];
    dispatch_vec_row<T, ADJ>(a, vals, row, lane, wred, d0, d1);
  }
  if (a.want_dots) grid_reduce2(d0, d1, a.partials, a.counter, a.dots_out, part_base, total);
}

// Multivectors: one launch per block-size class; rows [w0, w1) of the
// class-ordered row list all have block size R (R == 0: any size > 8).
template <typename T, int R, bool ADJ>
__global__ void __launch_bounds__(kThreads) apply_mv_kernel(ApplyArgs a, const T* __restrict__ vals, int w0, int w1,
                                                            int lpr, int G, int part_base, int total) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double d0 = 0.0, d1 = 0.0;
  for (int w = w0 + blockIdx.x * kWarps + warp; w < w1; w += gridDim.x * kWarps) {
    const int row = a.order[w];
    double r0 = 0.0, r1 = 0.0;
    if constexpr (R > 0) {
      mv_rows<T, R, ADJ>(a, vals, row, lane, lpr, G, 0, R, R, r0, r1);
    } else {
      const int r = a.bsz[row];
      for (int o0 = 0; o0 < r; o0 += 8)
        mv_rows<T, 8, ADJ>(a, vals, row, lane, lpr, G, o0, min(8, r - o0), r, r0, r1);
    }
    if (a.want_dots) {
      if (a.row_dots) {
        write_row_dots(a.row_dots, row, r0, r1);
      } else {
        d0 += r0;
        d1 += r1;
      }
    }
  }
  if (a.want_dots && !a.row_dots) grid_reduce2(d0, d1, a.partials, a.counter, a.dots_out, part_base, total);
}

// ------------------------------------------------ pipelined multivector apply
#include "vbg_pipe.cuh"
#include "vbg_tile.cuh"
#include "vbg_chain.cuh"
// Forward vectors on matrices whose blocks are all at most 8 x 8, every row
// from the slot records (vec_row_meta): a kernel of its own so that its
// register budget is not set by the general row paths: with 36 warps per
// SM every block row of a 5000-row matrix has its warp resident at once
// instead of some warps taking a second row after the first.  FP64 rows
// stage six columns at a time and complex rows four (kMetaCh), which keeps
// them inside this budget without spills.
constexpr int kMetaWarps = 4;  // warps of a record-driven vector CTA
template <typename T>
constexpr int kMetaCtas = 9;  // CTAs per SM
template <typename T>
constexpr int kMetaCh = std::is_same<T, cplx>::value ? 4 : std::is_same<T, double>::value ? 6 : 8;
template <typename T>
__global__ void __launch_bounds__(kMetaWarps * 32, kMetaCtas<T>) apply_vec_meta_kernel(ApplyArgs a,
                                                                                       const T* __restrict__ vals,
                                                                                       int part_base, int total) {
  __shared__ T wred_all[kMetaWarps * 32];
  if (a.npf && threadIdx.x == 0)
    for (int r = 0; r < a.npf; ++r) prefetch_share_l2(a.pf_ptr[r], a.pf_bytes[r]);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  T* wred = wred_all + warp * 32;
  double d0 = 0.0, d1 = 0.0;
  for (int w = blockIdx.x * kMetaWarps + warp; w < a.n_rows; w += gridDim.x * kMetaWarps)
    (void)dispatch_vec_row_meta<T, kMetaCh<T>>(a, vals, w, lane, wred, d0, d1);
  if (a.want_dots) grid_reduce2(d0, d1, a.partials, a.counter, a.dots_out, part_base, total);
}

template <typename T>
static int vec_meta_max_grid() {
  static int cached[kMaxDevices] = {};
  const int dev = current_device();
  if (!cached[dev]) {
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, apply_vec_meta_kernel<T>, kMetaWarps * 32, 0) !=
            cudaSuccess ||
        per_sm < 1)
      per_sm = 1;
    cached[dev] = per_sm * sm_count();
  }
  return cached[dev];
}

template <typename T, bool ADJ>
static int vec_max_grid() {
  static int cached[kMaxDevices] = {};
  const int dev = current_device();
  if (!cached[dev]) {
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, apply_vec_kernel<T, ADJ>, kThreads, 0) != cudaSuccess ||
        per_sm < 1)
      per_sm = 1;
    cached[dev] = per_sm * sm_count();
  }
  return cached[dev];
}

template <typename T, int R, bool ADJ>
static int mv_max_grid() {
  static int cached[kMaxDevices] = {};
  const int dev = current_device();
  if (!cached[dev]) {
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, apply_mv_kernel<T, R, ADJ>, kThreads, 0) !=
            cudaSuccess ||
        per_sm < 1)
      per_sm = 1;
    cached[dev] = per_sm * sm_count();
  }
  return cached[dev];
}

// Largest number of CTAs one apply (all class launches together) can use.
static int max_total_ctas() { return sm_count() * 8 * 10; }

// A launch that reduces its dots through `partials` must fit them: `total`
// CTAs of this apply against the room the caller gave (a.max_ctas), else the
// library's scratch (max_total_ctas()).
static int check_dot_ctas(const ApplyArgs& a, int total) {
  if (!a.want_dots || a.row_dots) return 0;
  const int cap = a.max_ctas > 0 ? a.max_ctas : max_total_ctas();
  if (total <= cap) return 0;
  return fail(a.max_ctas > 0 ? VBG_E_ARG : VBG_E_STATE,
              "this launch needs " + std::to_string(total) + " CTA partial sums; the dot scratch holds " +
                  std::to_string(cap));
}

// Working sets up to this size are prefetched into L2 by the vector apply.
constexpr long long kVecPrefetchMax = 32ll << 20;

// ------------------------------------------------------ scalar-row vectors
// Forward vectors on blocks of at most 8 x 8 with S consecutive threads per
// scalar output row: thread s of row i takes the blocks s, s + S, ... of
// i's block row -- its own row of each block (contiguous values) against
// the block column's X -- the S partial sums meet by shuffles and the first
// thread runs the epilogue on output i, so the epilogue's loads and stores
// are coalesced.  srow[i] holds i's slot range and its row inside the block,
// so a thread is one dependent load from its block list.  Against a warp per
// block row this issues far fewer instructions per row on small blocks (no
// per-block shuffles, no shared-memory reduction of partial rows).
constexpr int kSrowThreads = 256;
constexpr int kSrowCtas = 5;  // per SM (at most 51 registers)
template <typename T>
constexpr int kSrowCh = std::is_same<T, cplx>::value ? 4 : 8;

// ADJ: the adjoint over the column view -- a thread of output (scalar
// column) j takes the blocks of j's block column, reads the block's column
// (stride: its columns) conjugated against X over the block's rows;
// a.srow, a.slot_meta and a.blk_off then hold the scalar-column records and
// the column view's entry records and value offsets.
template <typename T, int S, bool ADJ = false>
__global__ void __launch_bounds__(kSrowThreads, kSrowCtas) apply_vec_srow_kernel(ApplyArgs a,
                                                                                 const T* __restrict__ vals,
                                                                                 int part_base, int total) {
  constexpr int CH = kSrowCh<T>;
  const T* __restrict__ x = static_cast<const T*>(a.X);
  const int lane = threadIdx.x & 31;
  const int64_t nt = a.n_scal * S;
  const int64_t stride = (int64_t)gridDim.x * kSrowThreads;
  double d0 = 0.0, d1 = 0.0;
  // warp-uniform trip count (the shuffles below need every lane)
  for (int64_t base = (int64_t)blockIdx.x * kSrowThreads + (threadIdx.x - lane); base < nt; base += stride) {
    const int64_t t = base + lane;
    const bool on = t < nt;
    const int64_t i = t / S;
    const int sl = (int)(t & (S - 1));
    T acc = zero_s<T>();
    if (on) {
      const int2 rec = __ldg(a.srow + i);
      const int o = rec.y & 0xff;
      const int e1 = rec.x + (rec.y >> 8);
      for (int e = rec.x + sl; e < e1; e += S) {
        const int2 mt = __ldg(a.slot_meta + e);
        const long long vo = __ldg(a.blk_off + e);
        const int nb = mt.y & 0xff;  // block columns
        const int jc = ADJ ? mt.y >> 8 : nb;  // inner length: the block's rows (ADJ) or columns
        const T* __restrict__ ap = vals + vo + (ADJ ? (long long)o : (long long)o * jc);
        const int st = ADJ ? nb : 1;
        const T* __restrict__ xp = x + (unsigned)mt.x;
        for (int q0 = 0; q0 < jc; q0 += CH) {
          T av[CH], xv[CH];
#pragma unroll
          for (int q = 0; q < CH; ++q) {
            av[q] = q0 + q < jc ? ap[(q0 + q) * st] : zero_s<T>();
            if (ADJ) av[q] = conj_s(av[q]);
            xv[q] = q0 + q < jc ? xp[q0 + q] : zero_s<T>();
          }
#pragma unroll
          for (int q = 0; q < CH; ++q) acc = fma_s(av[q], xv[q], acc);
        }
      }
    }
#pragma unroll
    for (int off = S / 2; off > 0; off >>= 1) acc = add_s(acc, shfl_xor_s(acc, off));
    if (on && sl == 0) {
      const T y = epi_value(a, acc, i);
      static_cast<T*>(a.Y)[i] = y;
      epi_finish(a, y, i, d0, d1);
    }
  }
  if (a.want_dots) grid_reduce2(d0, d1, a.partials, a.counter, a.dots_out, part_base, total);
}

__global__ void build_srow_kernel(int n, const int* __restrict__ ptr, const int* __restrict__ bsz,
                                  const int64_t* __restrict__ scal_off, int2* __restrict__ srow) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
    const int e0 = ptr[r], cnt = ptr[r + 1] - e0, b = bsz[r];
    const int64_t so = scal_off[r];
    for (int o = 0; o < b; ++o) srow[so + o] = make_int2(e0, (cnt << 8) | o);
  }
}

__global__ void build_scol_kernel(int n, const int* __restrict__ cptr, const int* __restrict__ cslot,
                                  const int* __restrict__ crow, const int* __restrict__ bsz,
                                  const int64_t* __restrict__ scal_off, const int64_t* __restrict__ blk_off,
                                  int2* __restrict__ scol, int2* __restrict__ cmeta, int64_t* __restrict__ cboff) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
    const int e0 = cptr[j], e1 = cptr[j + 1], c = bsz[j];
    for (int e = e0; e < e1; ++e) {
      const int i = crow[e];
      cmeta[e] = make_int2((int)scal_off[i], (bsz[i] << 8) | c);
      cboff[e] = blk_off[cslot[e]];
    }
    const int64_t so = scal_off[j];
    for (int o = 0; o < c; ++o) scol[so + o] = make_int2(e0, ((e1 - e0) << 8) | o);
  }
}

// Threads per scalar row of the scalar-row vector apply: option
// "apply.vec_lanes" (0 = by size, the default: the fewest of 1, 2, 4, 8 that
// give every SM 1024 threads; 1, 2, 4 or 8 fixed).
static std::atomic<int> g_opt_vec_lanes{0};
// Forward vector kernel: option "apply.vec_kernel" (0 = the autotuner's
// choice, the default; 1 = a warp per block row; 2 = scalar rows).
static std::atomic<int> g_opt_vec_kernel{0};

static int srow_lanes(const vbg_matrix* m) {
  const int opt = g_opt_vec_lanes.load(std::memory_order_relaxed);
  if (opt > 0) return opt;
  const int64_t want = (int64_t)sm_count() * 1024;
  int S = 1;
  while (S < 8 && m->N * S < want) S *= 2;
  return S;
}

// Whether the scalar-row kernel can run this matrix's forward vector applies
// (blocks of at most 8 x 8, the slot records in use, its thread count in
// range).
static bool srow_possible(const vbg_matrix* m) {
  return g_opt_vec_kernel.load(std::memory_order_relaxed) != 1 && m->max_bs <= 8 && m->n > 0 &&
         m->N <= (int64_t)INT32_MAX / 8;
}

// The scalar-row records when the scalar-row apply can run this forward
// vector apply (else nullptr): blocks of at most 8 x 8, the slot records in
// use, fewer than 2^23 slots in every block row; built on first use, never
// while the stream is being captured or when the caller allows no
// allocation.
static int vec_srow(const vbg_matrix* cm, cudaStream_t s, bool allow_alloc, const int2** out) {
  *out = nullptr;
  auto* m = const_cast<vbg_matrix*>(cm);
  if (!srow_possible(m)) return 0;
  if (!m->srow_valid) {
    if (!allow_alloc) return 0;
    cudaStreamCaptureStatus st;
    if (cudaStreamIsCapturing(s, &st) != cudaSuccess || st != cudaStreamCaptureStatusNone) return 0;
    if (m->nnzb >= (1ll << 23)) {
      if (!m->host_struct) return 0;
      for (int r = 0; r < m->n; ++r)
        if (m->h_row_ptr[r + 1] - m->h_row_ptr[r] >= (1 << 23)) return 0;
    }
    int rc = m->srow.ensure(std::max<int64_t>(m->N, 1) * sizeof(int2), s);
    if (rc) return rc;
    const int grid = std::max(1, std::min((m->n + 255) / 256, sm_count() * 8));
    build_srow_kernel<<<grid, 256, 0, s>>>(m->n, m->row_ptr.as<int>(), m->bsz.as<int>(), m->scal_off.as<int64_t>(),
                                           m->srow.as<int2>());
    VBG_CUDA(cudaGetLastError());
    m->srow_valid = true;
  }
  *out = m->srow.as<int2>();
  return 0;
}

// The adjoint's scalar-column records (see vec_srow), after the column view.
static int vec_scol(const vbg_matrix* cm, cudaStream_t s, bool allow_alloc, const int2** out) {
  *out = nullptr;
  auto* m = const_cast<vbg_matrix*>(cm);
  if (!srow_possible(m) || m->nnzb >= (1ll << 23) || m->N >= (int64_t)INT32_MAX) return 0;
  if (!m->scol_valid) {
    if (!allow_alloc) return 0;
    cudaStreamCaptureStatus st;
    if (cudaStreamIsCapturing(s, &st) != cudaSuccess || st != cudaStreamCaptureStatusNone) return 0;
    int rc;
    if ((rc = ensure_csc(m, s))) return rc;
    if ((rc = m->scol.ensure(std::max<int64_t>(m->N, 1) * sizeof(int2), s))) return rc;
    if ((rc = m->csc_meta.ensure(std::max<int64_t>(m->nnzb, 1) * sizeof(int2), s))) return rc;
    if ((rc = m->csc_boff.ensure(std::max<int64_t>(m->nnzb, 1) * sizeof(int64_t), s))) return rc;
    const int grid = std::max(1, std::min((m->n + 255) / 256, sm_count() * 8));
    build_scol_kernel<<<grid, 256, 0, s>>>(m->n, m->csc_ptr.as<int>(), m->csc_slot.as<int>(), m->csc_row.as<int>(),
                                           m->bsz.as<int>(), m->scal_off.as<int64_t>(), m->blk_off.as<int64_t>(),
                                           m->scol.as<int2>(), m->csc_meta.as<int2>(), m->csc_boff.as<int64_t>());
    VBG_CUDA(cudaGetLastError());
    m->scol_valid = true;
  }
  *out = m->scol.as<int2>();
  return 0;
}

template <typename T, int S, bool ADJ>
static int srow_max_grid() {
  static int cached[kMaxDevices] = {};
  const int dev = current_device();
  if (!cached[dev]) {
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, apply_vec_srow_kernel<T, S, ADJ>, kSrowThreads, 0) !=
            cudaSuccess ||
        per_sm < 1)
      per_sm = 1;
    cached[dev] = per_sm * sm_count();
  }
  return cached[dev];
}

template <typename T, int S, bool ADJ>
static int launch_vec_srow_s(const ApplyArgs& a, const T* vals, cudaStream_t s) {
  const int64_t want = (a.n_scal * S + kSrowThreads - 1) / kSrowThreads;
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(want, srow_max_grid<T, S, ADJ>()));
  if (int rc = check_dot_ctas(a, grid)) return rc;
  apply_vec_srow_kernel<T, S, ADJ><<<grid, kSrowThreads, 0, s>>>(a, vals, 0, grid);
  VBG_CUDA(cudaGetLastError());
  return 0;
}

template <typename T, bool ADJ>
static int launch_vec_srow(const vbg_matrix* m, const ApplyArgs& a0, const T* vals, cudaStream_t s) {
  ApplyArgs a = a0;
  if (ADJ) {
    a.slot_meta = m->csc_meta.as<int2>();
    a.blk_off = m->csc_boff.as<int64_t>();
  }
  switch (srow_lanes(m)) {
    case 1: return launch_vec_srow_s<T, 1, ADJ>(a, vals, s);
    case 2: return launch_vec_srow_s<T, 2, ADJ>(a, vals, s);
    case 4: return launch_vec_srow_s<T, 4, ADJ>(a, vals, s);
    default: return launch_vec_srow_s<T, 8, ADJ>(a, vals, s);
  }
}

template <typename T, bool ADJ>
static int launch_vec_t(const vbg_matrix* m, const ApplyArgs& a0, const T* vals, cudaStream_t s) {
  if (a0.srow) return launch_vec_srow<T, ADJ>(m, a0, vals, s);
  const bool meta_only = !ADJ && a0.slot_meta && m->max_bs <= 8;
  const int wpc = meta_only ? kMetaWarps : kWarps;
  int grid = (a0.n_rows + wpc - 1) / wpc;
  grid = std::max(1, std::min(grid, meta_only ? vec_meta_max_grid<T>() : vec_max_grid<T, ADJ>()));
  if (int rc = check_dot_ctas(a0, grid)) return rc;
  ApplyArgs a = a0;
  if (!ADJ && a.slot_meta) {
    const void* ptrs[4] = {vals, a.slot_meta, a.blk_off, a.X};
    const long long bytes[4] = {m->nnz * (long long)sizeof(T), m->nnzb * 8ll, m->nnzb * 8ll,
                                m->N * (long long)sizeof(T)};
    long long total = 0;
    for (int r = 0; r < 4; ++r) total += bytes[r];
    a.npf = 0;
    if (total <= kVecPrefetchMax)
      for (int r = 0; r < 4; ++r)
        if (bytes[r] >= 16 && reinterpret_cast<uintptr_t>(ptrs[r]) % 16 == 0) {
          a.pf_ptr[a.npf] = ptrs[r];
          a.pf_bytes[a.npf++] = bytes[r];
        }
  }
  if (meta_only)
    apply_vec_meta_kernel<T><<<grid, kMetaWarps * 32, 0, s>>>(a, vals, 0, grid);
  else
    apply_vec_kernel<T, ADJ><<<grid, kThreads, 0, s>>>(a, vals, 0, grid);
  VBG_CUDA(cudaGetLastError());
  return 0;
}

template <typename T, int R, bool ADJ>
static int launch_mv_class(const ApplyArgs& a, const T* vals, int w0, int w1, int lpr, int G, int grid, int base,
                           int total, cudaStream_t s) {
  apply_mv_kernel<T, R, ADJ><<<grid, kThreads, 0, s>>>(a, vals, w0, w1, lpr, G, base, total);
  VBG_CUDA(cudaGetLastError());
  return 0;
}

template <typename T, bool ADJ>
static int mv_class_grid(int r, int rows) {
  int cap;
  switch (r) {
    case 1: cap = mv_max_grid<T, 1, ADJ>(); break;
    case 2: cap = mv_max_grid<T, 2, ADJ>(); break;
    case 3: cap = mv_max_grid<T, 3, ADJ>(); break;
    case 4: cap = mv_max_grid<T, 4, ADJ>(); break;
    case 5: cap = mv_max_grid<T, 5, ADJ>(); break;
    case 6: cap = mv_max_grid<T, 6, ADJ>(); break;
    case 7: cap = mv_max_grid<T, 7, ADJ>(); break;
    case 8: cap = mv_max_grid<T, 8, ADJ>(); break;
    default: cap = mv_max_grid<T, 0, ADJ>(); break;
  }
  return std::max(1, std::min((rows + kWarps - 1) / kWarps, cap));
}

template <typename T, bool ADJ>
static int launch_mv_t(const vbg_matrix* m, const ApplyArgs& a, const T* vals, cudaStream_t s) {
  const int nvec = a.ld / VT<T>::E;
  int lpr = nvec >= 32 ? 32 : nvec;
  int G = 32 / lpr;
  if (G > 1 && (lpr & (lpr - 1))) G = 1;  // butterflies need power-of-two groups
  // class segments of the class-ordered row list; rows > 8 share one launch
  std::vector<std::tuple<int, int, int>> segs;  // (R template, w0, w1)
  for (const auto& cs : m->class_segs) {
    const int rt = cs.r <= 8 ? cs.r : 0;
    if (!segs.empty() && rt == 0 && std::get<0>(segs.back()) == 0)
      std::get<2>(segs.back()) = cs.w1;
    else
      segs.emplace_back(rt, cs.w0, cs.w1);
  }
  std::vector<int> grids;
  int total = 0;
  for (auto& sg : segs) {
    grids.push_back(mv_class_grid<T, ADJ>(std::get<0>(sg), std::get<2>(sg) - std::get<1>(sg)));
    total += grids.back();
  }
  if (int rc = check_dot_ctas(a, total)) return rc;
  int base = 0;
  for (size_t i = 0; i < segs.size(); ++i) {
    const int w0 = std::get<1>(segs[i]), w1 = std::get<2>(segs[i]);
    int rc = 0;
    switch (std::get<0>(segs[i])) {
      case 1: rc = launch_mv_class<T, 1, ADJ>(a, vals, w0, w1, lpr, G, grids[i], base, total, s); break;
      case 2: rc = launch_mv_class<T, 2, ADJ>(a, vals, w0, w1, lpr, G, grids[i], base, total, s); break;
      case 3: rc = launch_mv_class<T, 3, ADJ>(a, vals, w0, w1, lpr, G, grids[i], base, total, s); break;
      case 4: rc = launch_mv_class<T, 4, ADJ>(a, vals, w0, w1, lpr, G, grids[i], base, total, s); break;
      case 5: rc = launch_mv_class<T, 5, ADJ>(a, vals, w0, w1, lpr, G, grids[i], base, total, s); break;
      case 6: rc = launch_mv_class<T, 6, ADJ>(a, vals, w0, w1, lpr, G, grids[i], base, total, s); break;
      case 7: rc = launch_mv_class<T, 7, ADJ>(a, vals, w0, w1, lpr, G, grids[i], base, total, s); break;
      case 8: rc = launch_mv_class<T, 8, ADJ>(a, vals, w0, w1, lpr, G, grids[i], base, total, s); break;
      default: rc = launch_mv_class<T, 0, ADJ>(a, vals, w0, w1, lpr, G, grids[i], base, total, s); break;
    }
    if (rc) return rc;
    base += grids[i];
  }
  return 0;
}

// Whether apply_pipe_kernel handles this (forward) multivector apply: blocks
// at most 8 x 8, rows a whole number of warp widths, buffers aligned to the
// per-lane piece.
// Lane groups of apply_pipe_kernel for leading dimension ld: 1 when a row
// of X is at least a warp of pieces wide, 2 or 4 for narrower rows, 0 when
// ld is no whole number of group widths.
template <typename T>
static int pipe_groups(int ld) {
  constexpr int EV = PipeEV<T>::v;
  if (ld % (32 * EV) == 0) return 1;
  if (ld % (16 * EV) == 0) return 2;
  if (ld % (8 * EV) == 0) return 4;
  return 0;
}

template <typename T>
static bool pipe_eligible(const vbg_matrix* m, bool adj, const ApplyArgs& a) {
  constexpr int EV = PipeEV<T>::v;
  constexpr uintptr_t LB = EV * sizeof(T);
  if (adj || a.ld <= 1 || m->max_bs < 1 || m->max_bs > kPipeMaxBs || pipe_groups<T>(a.ld) == 0) return false;
  if (m->N >= (int64_t)INT32_MAX || !a.slot_meta) return false;
  if (reinterpret_cast<uintptr_t>(a.X) % 16) return false;  // bulk copies of X rows
  const void* ptrs[5] = {a.X, a.Xprev, a.Y, a.dotw, a.acc};
  for (const void* p : ptrs)
    if (p && reinterpret_cast<uintptr_t>(p) % LB) return false;
  return true;
}

// X rows per span (and per stage of the ring): at least the largest block.
static int pipe_span_cap(const vbg_matrix* m) { return std::max(m->max_bs, std::min(kPipeSpanCap, kPipeMaxBs)); }

// Grid and dynamic shared memory of apply_pipe_kernel<T, EV, G> for this apply.
template <typename T, int G>
static int pipe_grid_g(const vbg_matrix* m, const ApplyArgs& a, int* grid, size_t* smem) {
  constexpr int EV = PipeEV<T>::v;
  static bool attr_set[kMaxDevices] = {};
  static int per_sm_dev[kMaxDevices][kPipeMaxBs + 1] = {};
  const int dev = current_device();
  int* per_sm = per_sm_dev[dev];
  const int cm = pipe_span_cap(m);
  *smem = kPipeWarps * pipe_warp_bytes<T, G>(cm);
  if (!attr_set[dev]) {
    VBG_CUDA(cudaFuncSetAttribute(apply_pipe_kernel<T, EV, G>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)(kPipeWarps * pipe_warp_bytes<T, G>(kPipeMaxBs))));
    attr_set[dev] = true;
  }
  if (!per_sm[cm]) {
    int b = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, apply_pipe_kernel<T, EV, G>, kPipeWarps * 32, *smem) !=
            cudaSuccess ||
        b < 1)
      b = 1;
    per_sm[cm] = b;
  }
  const int nitems = ((a.n_rows + kPipeRows - 1) / kPipeRows) * (a.ld / (PipeShape<G>::L * EV));
  *grid = std::max(1, std::min((nitems + kPipeWarps - 1) / kPipeWarps, per_sm[cm] * sm_count()));
  return 0;
}

template <typename T>
static int pipe_grid(const vbg_matrix* m, const ApplyArgs& a, int* grid, size_t* smem) {
  switch (pipe_groups<T>(a.ld)) {
    case 1: return pipe_grid_g<T, 1>(m, a, grid, smem);
    case 2: return pipe_grid_g<T, 2>(m, a, grid, smem);
    default: return pipe_grid_g<T, 4>(m, a, grid, smem);
  }
}

// Whether this apply runs on apply_pipe_kernel: eligible, and the kernel
// layout of the values exists or may be built here (never while the stream
// is being captured, nor when the caller allows no allocation).
template <typename T>
static bool pipe_use(const vbg_matrix* m, bool adj, const ApplyArgs& a, cudaStream_t s, bool allow_alloc) {
  if (!pipe_eligible<T>(m, adj, a)) return false;
  constexpr bool f32 = std::is_same<T, float>::value;
  if ((f32 ? m->valsK32_valid : m->valsK_valid) && m->span_cap == pipe_span_cap(m)) return true;
  if (!allow_alloc) return false;
  cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(s, &st) != cudaSuccess || st != cudaStreamCaptureStatusNone) return false;
  return ensure_kernel_layout(m, f32, s) == 0 && ensure_spans(m, pipe_span_cap(m), s) == 0;
}

template <typename T, int G>
static int launch_pipe_g(const vbg_matrix* m, const ApplyArgs& a0, cudaStream_t s) {
  constexpr int EV = PipeEV<T>::v;
  constexpr bool f32 = std::is_same<T, float>::value;
  int grid = 0;
  size_t smem = 0;
  int rc = pipe_grid_g<T, G>(m, a0, &grid, &smem);
  if (rc) return rc;
  if ((rc = check_dot_ctas(a0, grid))) return rc;
  ApplyArgs a = a0;
  a.koff = (f32 ? m->koff32 : m->koff).as<int64_t>();
  a.spans = m->spans.as<int4>();
  a.span_koff32 = m->span_koff32.as<int64_t>();
  a.row_sptr = m->row_sptr.as<int>();
  const T* vals = (f32 ? m->valsK32 : m->valsK).as<T>();
  apply_pipe_kernel<T, EV, G><<<grid, kPipeWarps * 32, smem, s>>>(a, vals, m->span_cap,
                                                                 a.ld / (PipeShape<G>::L * EV), 0, grid);
  VBG_CUDA(cudaGetLastError());
  return 0;
}

template <typename T>
static int launch_pipe_t(const vbg_matrix* m, const ApplyArgs& a, cudaStream_t s) {
  switch (pipe_groups<T>(a.ld)) {
    case 1: return launch_pipe_g<T, 1>(m, a, s);
    case 2: return launch_pipe_g<T, 2>(m, a, s);
    default: return launch_pipe_g<T, 4>(m, a, s);
  }
}

// Whether this apply runs on apply_tile_kernel<T, EV, G>: a row of X is
// 32 / G lanes of EV scalars (ld = 32 / G * EV: FP64 and FP32 at 64
// columns with EV = 2, complex and FP32 at 32 with EV = 1, FP64 and FP32 at
// 16 with EV = 1 and G = 2 lane groups), the pipelined apply's value layout
// applies, the bulk-copied rows (X, Xprev, the dot partner) start on 16-byte
// boundaries, and the matrix has a tile plan for it (built here unless
// capturing or allocation is not allowed).
// Largest tile height (block rows) of the tiled applies at this leading
// dimension and value size: the autotuner's choice, kTileRowsMax before it.
static int tile_cap(const vbg_matrix* m, int ld, int es) {
  auto it = m->tile_rows_cap.find(std::make_pair(ld, es));
  return it == m->tile_rows_cap.end() ? kTileRowsMax : it->second;
}

// Whether the tiled kernel takes its tiles from the plan's work queue (the
// autotuner's choice) or in a fixed stride (default).
static bool tile_queue_on(const vbg_matrix* m, int ld, int es) {
  auto it = m->tile_queue.find(std::make_pair(ld, es));
  return it != m->tile_queue.end() && it->second != 0;
}

template <typename T, int EV = PipeEV<T>::v, int G = 1>
static bool tile_use(const vbg_matrix* m, bool adj, const ApplyArgs& a, cudaStream_t s, bool allow_alloc,
                     TilePlan** plan) {
  *plan = nullptr;
  if (a.ld != 32 / G * EV || !pipe_use<T>(m, adj, a, s, allow_alloc)) return false;
  const void* copied[3] = {a.X, a.Xprev, a.dotw};
  for (const void* p : copied)
    if (p && reinterpret_cast<uintptr_t>(p) % 16) return false;
  const int rb = 32 / G * EV * (int)sizeof(T);
  const int cap = tile_cap(m, a.ld, (int)sizeof(T));
  auto it = m->tile_plans.find(std::make_tuple(rb, (int)sizeof(T), cap));
  if (it != m->tile_plans.end()) {
    if (it->second->rows > 0) *plan = it->second.get();
    return *plan != nullptr;
  }
  if (!allow_alloc) return false;
  cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(s, &st) != cudaSuccess || st != cudaStreamCaptureStatusNone) return false;
  return tile_plan(m, rb, (int)sizeof(T), s, plan, cap) == 0 && *plan != nullptr;
}

// Grid of apply_tile_kernel<T, EV, G> for a plan: the CTAs resident at once,
// at most one per tile.
template <typename T, int EV, int G = 1>
static int tile_grid(TilePlan* plan, int* grid) {
  static bool attr_set[kMaxDevices] = {};
  const int dev = current_device();
  if (!attr_set[dev]) {
    VBG_CUDA(cudaFuncSetAttribute(apply_tile_kernel<T, EV, G>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)kTileSmemBudget));
    attr_set[dev] = true;
  }
  if (!plan->grid) {
    int b = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, apply_tile_kernel<T, EV, G>, kTileWarps * 32, plan->smem) !=
            cudaSuccess ||
        b < 1)
      b = 1;
    plan->grid = std::max(1, std::min(plan->ntiles, b * sm_count()));
  }
  *grid = plan->grid;
  return 0;
}

template <typename T, int EV = PipeEV<T>::v, int G = 1>
static int launch_tile(const vbg_matrix* m, const ApplyArgs& a0, TilePlan* plan, cudaStream_t s) {
  constexpr bool f32 = std::is_same<T, float>::value;
  int grid = 0;
  int rc = tile_grid<T, EV, G>(plan, &grid);
  if (rc) return rc;
  if ((rc = check_dot_ctas(a0, grid))) return rc;
  ApplyArgs a = a0;
  a.koff = (f32 ? m->koff32 : m->koff).as<int64_t>();
  a.spans = m->spans.as<int4>();
  a.span_koff32 = m->span_koff32.as<int64_t>();
  a.row_sptr = m->row_sptr.as<int>();
  const T* vals = (f32 ? m->valsK32 : m->valsK).as<T>();
  apply_tile_kernel<T, EV, G><<<grid, kTileWarps * 32, plan->smem, s>>>(
      a, vals, plan->tiles.as<int4>(), plan->ranges.as<int4>(), plan->qidx.as<unsigned short>(),
      plan->rowinfo.as<int4>(), plan->ntiles, (unsigned)tile_vals_bytes(plan->vcap, (int)sizeof(T)),
      (unsigned)plan->qcap, tile_queue_on(m, a.ld, (int)sizeof(T)) ? plan->queue.as<int>() : nullptr, 0, grid);
  VBG_CUDA(cudaGetLastError());
  return 0;
}

// Whether this apply runs on apply_chain_kernel<T, EV, G>: the tiled
// apply's conditions, and the matrix has a chain plan (built here unless
// capturing or allocation is not allowed).
template <typename T, int EV = PipeEV<T>::v, int G = 1>
static bool chain_use(const vbg_matrix* m, const ApplyArgs& a, cudaStream_t s, bool allow_alloc, ChainPlan** plan) {
  *plan = nullptr;
  if (g_opt_chain.load(std::memory_order_relaxed) == 0) return false;
  if (a.ld != 32 / G * EV || !pipe_use<T>(m, false, a, s, allow_alloc)) return false;
  const void* aligned[3] = {a.X, a.Xprev, a.dotw};
  for (const void* p : aligned)
    if (p && reinterpret_cast<uintptr_t>(p) % 16) return false;
  const int rb = 32 / G * EV * (int)sizeof(T);
  auto it = m->chain_plans.find(std::make_pair(rb, (int)sizeof(T)));
  if (it != m->chain_plans.end()) {
    if (it->second->rows > 0) *plan = it->second.get();
    return *plan != nullptr;
  }
  if (!allow_alloc) return false;
  cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(s, &st) != cudaSuccess || st != cudaStreamCaptureStatusNone) return false;
  return chain_plan(m, rb, (int)sizeof(T), s, plan) == 0 && *plan != nullptr;
}

template <typename T, int EV = PipeEV<T>::v, int G = 1>
static int launch_chain(const vbg_matrix* m, const ApplyArgs& a0, ChainPlan* plan, cudaStream_t s) {
  constexpr bool f32 = std::is_same<T, float>::value;
  static bool attr_set[kMaxDevices] = {};
  const int dev = current_device();
  if (!attr_set[dev]) {
    VBG_CUDA(cudaFuncSetAttribute(apply_chain_kernel<T, EV, G>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)kChainSmemBudget));
    attr_set[dev] = true;
  }
  const int grid = plan->nctas;
  int rc = check_dot_ctas(a0, grid);
  if (rc) return rc;
  ApplyArgs a = a0;
  a.koff = (f32 ? m->koff32 : m->koff).as<int64_t>();
  a.spans = m->spans.as<int4>();
  a.span_koff32 = m->span_koff32.as<int64_t>();
  a.row_sptr = m->row_sptr.as<int>();
  const T* vals = (f32 ? m->valsK32 : m->valsK).as<T>();
  apply_chain_kernel<T, EV, G><<<grid, (plan->rows + 1) * 32, plan->smem, s>>>(
      a, vals, plan->tiles.as<int4>(), plan->loads.as<int4>(), plan->cta_ptr.as<int>(), plan->qidx.as<unsigned short>(),
      plan->rowinfo.as<int4>(), plan->rows, (unsigned)tile_vals_bytes(plan->vcap, (int)sizeof(T)),
      (unsigned)plan->qcap, 0, grid);
  VBG_CUDA(cudaGetLastError());
  return 0;
}

// Builds the tile plan an apply with leading dimension ld would use (before
// a graph capture, which may not build it).  Real matrices only for f32.
static int tile_prepare(const vbg_matrix* m, bool f32, int ld, cudaStream_t s) {
  TilePlan* tp = nullptr;
  ChainPlan* cp = nullptr;
  int rb = 0, es = 0;
  if (f32) {
    if (ld != 16 && ld != 32 && ld != 64) return 0;
    rb = ld * 4;
    es = 4;
  } else if (m->dtype == VBG_C128) {
    if (ld != 32 * PipeEV<cplx>::v) return 0;
    rb = 32 * 16;
    es = 16;
  } else {
    if (ld != 16 && ld != 32 * PipeEV<double>::v) return 0;
    rb = ld * 8;
    es = 8;
  }
  if (chain_enabled(es)) {
    const int rc = chain_plan(m, rb, es, s, &cp);
    if (rc || cp) return rc;
  }
  return tile_plan(m, rb, es, s, &tp);
}

// Validates arguments and fills the structure part of ApplyArgs.
static int prepare(const vbg_matrix* m, bool adj, int k, int ld, ApplyArgs& a, cudaStream_t s) {
  VBG_CHECK(m, VBG_E_ARG, "null matrix");
  VBG_CHECK(k >= 1 && ld >= k, VBG_E_ARG, "invalid k / ld");
  std::memset(&a, 0, sizeof(a));
  a.n_rows = m->n;
  a.bsz = m->bsz.as<int>();
  a.scal_off = m->scal_off.as<int64_t>();
  a.blk_off = m->blk_off.as<int64_t>();
  a.ld = ld;
  a.alpha = 1.0;
  if (!adj) {
    a.order = m->row_perm.as<int>();
    a.ptr = m->row_ptr.as<int>();
    a.ent_slot = nullptr;
    a.ent_src = m->col_ind.as<int>();
    // the records hold 32-bit X offsets and 8-bit block sizes
    a.slot_meta = (m->N < (int64_t)INT32_MAX && m->max_bs <= 255) ? m->slot_meta.as<int2>() : nullptr;
  } else {
    int rc = ensure_csc(m, s);
    if (rc) return rc;
    a.order = m->row_perm.as<int>();
    a.ptr = m->csc_ptr.as<int>();
    a.ent_slot = m->csc_slot.as<int>();
    a.ent_src = m->csc_row.as<int>();
  }
  return 0;
}

// Forward multivector apply on kernel `which` (VBG_KERNEL_CHAIN, _TILE, _PIPE
// or _ROWS; -1: the default order -- chained tiles when the apply.chain
// option allows them, tiles, the pipelined kernel, rows).  Returns
// kNotApplicable when `which` cannot run this apply.
constexpr int kNotApplicable = 1;

template <typename T>
static int launch_fwd_mv(const vbg_matrix* m, const ApplyArgs& a, const T* v, cudaStream_t s, bool allow_alloc,
                         int which) {
  const bool any = which < 0;
  TilePlan* tp = nullptr;
  ChainPlan* cp = nullptr;
  if (any ? chain_enabled((int)sizeof(T)) : which == VBG_KERNEL_CHAIN) {
    if (chain_use<T>(m, a, s, allow_alloc, &cp)) return launch_chain<T>(m, a, cp, s);
    if constexpr (std::is_same<T, float>::value) {
      if (chain_use<float, 1>(m, a, s, allow_alloc, &cp)) return launch_chain<float, 1>(m, a, cp, s);
    }
    if constexpr (!std::is_same<T, cplx>::value) {
      if (chain_use<T, 1, 2>(m, a, s, allow_alloc, &cp)) return launch_chain<T, 1, 2>(m, a, cp, s);
    }
    if (!any) return kNotApplicable;
  }
  if (any || which == VBG_KERNEL_TILE) {
    if (tile_use<T>(m, false, a, s, allow_alloc, &tp)) return launch_tile<T>(m, a, tp, s);
    if constexpr (std::is_same<T, float>::value) {
      if (tile_use<float, 1>(m, false, a, s, allow_alloc, &tp)) return launch_tile<float, 1>(m, a, tp, s);
    }
    if constexpr (!std::is_same<T, cplx>::value) {
      if (tile_use<T, 1, 2>(m, false, a, s, allow_alloc, &tp)) return launch_tile<T, 1, 2>(m, a, tp, s);
    }
    if (!any) return kNotApplicable;
  }
  if (any || which == VBG_KERNEL_PIPE) {
    if (pipe_use<T>(m, false, a, s, allow_alloc)) return launch_pipe_t<T>(m, a, s);
    if (!any) return kNotApplicable;
  }
  return launch_mv_t<T, false>(m, a, v, s);
}

// The autotuner: the first forward multivector apply with a given leading
// dimension and precision on a matrix (outside a stream capture, with
// allocation allowed) times each kernel that can run it -- the chained
// tiles, the tiles at three tile heights (at most 16, 12 and 8 block rows,
// each its own plan) with their tiles in a fixed stride or from a work
// queue, the pipelined kernel -- three launches each after one
// untimed launch, on the caller's buffers (the trials write Y and the dots,
// which the real launch then overwrites; they leave the accumulator alone)
// and keeps the fastest kernel for the matrix (vbg_matrix::tuned) and the
// fastest tile height and order for its tiled kernel
// (vbg_matrix::tile_rows_cap, tile_queue).  Option
// "apply.autotune" (default 1) switches it off; an explicit "apply.chain" of
// 0 or 1 takes the kernel choice out of its hands.
static std::atomic<int> g_opt_autotune{1};

template <typename T>
static int autotune_fwd(const vbg_matrix* m, const ApplyArgs& a0, const T* v, cudaStream_t s, int* choice) {
  ApplyArgs a = a0;
  a.acc = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  VBG_CUDA(cudaEventCreate(&e0));
  cudaError_t ce = cudaEventCreate(&e1);
  if (ce != cudaSuccess) {
    cudaEventDestroy(e0);
    return cuda_fail(ce, "cudaEventCreate");
  }
  float best = 0.0f, best_tile = 0.0f;
  int rc = 0, best_cap = 0, best_queue = 0;
  *choice = -1;
  auto* mm = const_cast<vbg_matrix*>(m);
  const auto cap_key = std::make_pair(a.ld, (int)sizeof(T));
  for (int cand : {VBG_KERNEL_CHAIN, VBG_KERNEL_TILE, VBG_KERNEL_PIPE}) {
    // the tiled kernel once per tile height cap (its own plan each) and per
    // tile order (fixed stride, work queue)
    for (int trial = 0; trial < 6; ++trial) {
      const int cap = trial < 2 ? kTileRowsMax : trial < 4 ? 12 : 8;
      const int queue = trial & 1;
      if (cand != VBG_KERNEL_TILE && trial > 0) break;
      if (cand == VBG_KERNEL_TILE) {
        mm->tile_rows_cap[cap_key] = cap;
        mm->tile_queue[cap_key] = queue;
      }
      rc = launch_fwd_mv<T>(m, a, v, s, true, cand);
      if (rc == kNotApplicable) {
        rc = 0;
        break;
      }
      if (rc) break;
      cudaEventRecord(e0, s);
      for (int k = 0; k < 3 && !rc; ++k) rc = launch_fwd_mv<T>(m, a, v, s, true, cand);
      cudaEventRecord(e1, s);
      if (rc) break;
      if ((ce = cudaEventSynchronize(e1)) != cudaSuccess) {
        rc = cuda_fail(ce, "autotune");
        break;
      }
      float ms = 0.0f;
      cudaEventElapsedTime(&ms, e0, e1);
      if (cand == VBG_KERNEL_TILE && (best_cap == 0 || ms < best_tile)) {
        best_tile = ms;
        best_cap = cap;
        best_queue = queue;
      }
      if (*choice < 0 || ms < best) {
        best = ms;
        *choice = cand;
      }
    }
    if (cand == VBG_KERNEL_TILE) {
      mm->tile_rows_cap[cap_key] = best_cap ? best_cap : kTileRowsMax;
      mm->tile_queue[cap_key] = best_cap ? best_queue : 0;
    }
    if (rc) break;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (!rc && *choice < 0) *choice = VBG_KERNEL_ROWS;
  return rc;
}

// The kernel a forward multivector apply runs: the tuned choice when the
// autotuner may decide (tuning now if it has not), else -1 (default order).
template <typename T>
static int fwd_choice(const vbg_matrix* m, bool f32, const ApplyArgs& a, const T* v, cudaStream_t s,
                      bool allow_alloc, int* which) {
  *which = -1;
  if (!g_opt_autotune.load() || g_opt_chain.load() != 2) return 0;
  auto* mm = const_cast<vbg_matrix*>(m);
  const auto key = std::make_pair(a.ld, f32 ? 1 : 0);
  auto it = mm->tuned.find(key);
  if (it != mm->tuned.end()) {
    *which = it->second;
    return 0;
  }
  if (!allow_alloc) return 0;
  cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(s, &st) != cudaSuccess || st != cudaStreamCaptureStatusNone) return 0;
  int choice = -1;
  int rc = autotune_fwd<T>(m, a, v, s, &choice);
  if (rc) return rc;
  mm->tuned[key] = choice;
  *which = choice;
  return 0;
}

// Dispatch on scalar type / vector-vs-multivector.  `f32` selects the FP32
// shadow values (real matrices only).
// `allow_alloc` false: the call may not allocate device memory (the pipelined
// kernel then runs only if its value layout already exists).
// The forward vector kernel: a warp per block row (VBG_KERNEL_VECTOR) or the
// scalar-row kernel (VBG_KERNEL_SCALAR_ROWS; *srow_out set).  Option
// "apply.vec_kernel" forces one; at 0 the autotuner times both on the first
// vector apply per matrix and precision (three launches each, the
// accumulator off) and keeps the faster.  Untuned (autotuner off, no
// allocation allowed, or the stream being captured) complex values take the
// scalar-row kernel, real ones a warp per block row.
template <typename T, bool ADJ = false>
static int vec_kernel(const vbg_matrix* m, bool f32, const ApplyArgs& a0, const T* vals, cudaStream_t s,
                      bool allow_alloc, const int2** srow_out) {
  *srow_out = nullptr;
  const int2* sr = nullptr;
  if (int rc = ADJ ? vec_scol(m, s, allow_alloc, &sr) : vec_srow(m, s, allow_alloc, &sr)) return rc;
  if (!sr) return 0;
  if (g_opt_vec_kernel.load() == 2) {
    *srow_out = sr;
    return 0;
  }
  auto* mm = const_cast<vbg_matrix*>(m);
  // the adjoint's choice under its own key
  const auto key = std::make_pair(1, (f32 ? 1 : 0) + (ADJ ? 2 : 0));
  auto it = mm->tuned.find(key);
  if (it != mm->tuned.end()) {
    if (it->second == VBG_KERNEL_SCALAR_ROWS) *srow_out = sr;
    return 0;
  }
  cudaStreamCaptureStatus st;
  if (!g_opt_autotune.load() || !allow_alloc || cudaStreamIsCapturing(s, &st) != cudaSuccess ||
      st != cudaStreamCaptureStatusNone) {
    if (std::is_same<T, cplx>::value) *srow_out = sr;
    return 0;
  }
  ApplyArgs c[2];
  c[0] = a0;
  c[0].acc = nullptr;
  c[0].srow = nullptr;
  c[1] = c[0];
  c[1].srow = sr;
  c[1].n_scal = m->N;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  VBG_CUDA(cudaEventCreate(&e0));
  cudaError_t ce = cudaEventCreate(&e1);
  if (ce != cudaSuccess) {
    cudaEventDestroy(e0);
    return cuda_fail(ce, "cudaEventCreate");
  }
  float ms[2] = {0.0f, 0.0f};
  int rc = 0;
  for (int k = 0; k < 2 && !rc; ++k) {
    if ((rc = launch_vec_t<T, ADJ>(m, c[k], vals, s))) break;
    cudaEventRecord(e0, s);
    for (int r = 0; r < 3 && !rc; ++r) rc = launch_vec_t<T, ADJ>(m, c[k], vals, s);
    cudaEventRecord(e1, s);
    if (rc) break;
    if ((ce = cudaEventSynchronize(e1)) != cudaSuccess) {
      rc = cuda_fail(ce, "autotune");
      break;
    }
    cudaEventElapsedTime(&ms[k], e0, e1);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc) return rc;
  mm->tuned[key] = ms[1] < ms[0] ? VBG_KERNEL_SCALAR_ROWS : VBG_KERNEL_VECTOR;
  if (ms[1] < ms[0]) *srow_out = sr;
  return 0;
}

static int launch_apply(const vbg_matrix* m, bool adj, bool f32, const ApplyArgs& a_in, cudaStream_t s,
                        bool allow_alloc = true) {
  if (m->n == 0) return 0;
  const bool mv = a_in.ld > 1;
  ApplyArgs a = a_in;
  if (!mv && !adj && a.slot_meta && !a.row_dots) {
    int rc;
    a.n_scal = m->N;
    if (f32) {
      if ((rc = ensure_vals32(m, s))) return rc;
      rc = vec_kernel<float>(m, true, a, m->vals32.as<float>(), s, allow_alloc, &a.srow);
    } else if (m->dtype == VBG_C128) {
      rc = vec_kernel<cplx>(m, false, a, m->vals.as<cplx>(), s, allow_alloc, &a.srow);
    } else {
      rc = vec_kernel<double>(m, false, a, m->vals.as<double>(), s, allow_alloc, &a.srow);
    }
    if (rc) return rc;
  } else if (!mv && adj && !a.row_dots && m->N < (int64_t)INT32_MAX) {
    int rc;
    a.n_scal = m->N;
    if (f32) {
      if ((rc = ensure_vals32(m, s))) return rc;
      rc = vec_kernel<float, true>(m, true, a, m->vals32.as<float>(), s, allow_alloc, &a.srow);
    } else if (m->dtype == VBG_C128) {
      rc = vec_kernel<cplx, true>(m, false, a, m->vals.as<cplx>(), s, allow_alloc, &a.srow);
    } else {
      rc = vec_kernel<double, true>(m, false, a, m->vals.as<double>(), s, allow_alloc, &a.srow);
    }
    if (rc) return rc;
  }
  if (mv) {
    const size_t es = f32 ? 4 : elem_size(m->dtype);
    VBG_CHECK(((size_t)a.ld * es) % 16 == 0, VBG_E_ARG,
              "multivector leading dimension must span a multiple of 16 bytes");
  }
  auto fwd = [&](auto tag, const auto* v) -> int {
    using T = decltype(tag);
    int which = -1;
    int rc = fwd_choice<T>(m, f32, a, v, s, allow_alloc, &which);
    if (rc) return rc;
    rc = launch_fwd_mv<T>(m, a, v, s, allow_alloc, which);
    return rc == kNotApplicable ? launch_fwd_mv<T>(m, a, v, s, allow_alloc, -1) : rc;
  };
  if (f32) {
    int rc = ensure_vals32(m, s);
    if (rc) return rc;
    const float* v = m->vals32.as<float>();
    if (adj) return mv ? launch_mv_t<float, true>(m, a, v, s) : launch_vec_t<float, true>(m, a, v, s);
    return mv ? fwd(float{}, v) : launch_vec_t<float, false>(m, a, v, s);
  }
  if (m->dtype == VBG_C128) {
    const cplx* v = m->vals.as<cplx>();
    if (adj) return mv ? launch_mv_t<cplx, true>(m, a, v, s) : launch_vec_t<cplx, true>(m, a, v, s);
    return mv ? fwd(cplx{}, v) : launch_vec_t<cplx, false>(m, a, v, s);
  }
  const double* v = m->vals.as<double>();
  if (adj) return mv ? launch_mv_t<double, true>(m, a, v, s) : launch_vec_t<double, true>(m, a, v, s);
  return mv ? fwd(double{}, v) : launch_vec_t<double, false>(m, a, v, s);
}

// ------------------------------------------------------------ helpers

template <typename T>
__global__ void sumsq_kernel(const T* __restrict__ x, int64_t n, double* partials, unsigned* counter, double* out) {
  double d = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    d += re_dot(x[i], x[i]);
  grid_reduce2(d, 0.0, partials, counter, out, 0, gridDim.x);
}

__global__ void f64_to_f32_rows(const double* __restrict__ src, int64_t rows, int ld_src, float* __restrict__ dst,
                                int ld_dst) {
  const int64_t total = rows * ld_dst;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = i / ld_dst;
    const int c = (int)(i - r * ld_dst);
    dst[i] = c < ld_src ? (float)src[r * ld_src + c] : 0.0f;
  }
}

// dots[step] = (d0, d1) -> moments.  Batched: segment sg (one thread each)
// reads dots[step * stride + 2 * sg + {0, 1}] and writes mu[sg * M + n].
__global__ void kpm_finalize(const double* __restrict__ dots, int M, int two_moment, double* __restrict__ mu,
                             int stride, int nseg) {
  const int sg = blockIdx.x * blockDim.x + threadIdx.x;
  if (sg >= nseg) return;
  auto D = [&](int step, int w) { return dots[(size_t)step * stride + 2 * sg + w]; };
  double* out = mu + (size_t)sg * M;
  // step 0 = (sum |v0|^2, -), step 1 = the apply producing t_1, step n+1 = the one producing t_{n+1}
  const double mu0 = D(0, 0);
  out[0] = mu0;
  if (M < 2) return;
  const double mu1 = D(1, 0);
  out[1] = mu1;
  if (two_moment) {
    if (M > 2) out[2] = 2.0 * D(1, 1) - mu0;
    for (int n = 1;; ++n) {
      const int odd = 2 * n + 1, even = 2 * n + 2;
      if (odd >= M) break;
      out[odd] = 2.0 * D(n + 1, 0) - mu1;
      if (even < M) out[even] = 2.0 * D(n + 1, 1) - mu0;
    }
  } else {
    for (int n = 2; n < M; ++n) out[n] = D(n, 0);
  }
}

// Fixed-order sum of two values over the threads of a block (blockDim.x
// a multiple of 32, at most 1024); result in thread 0.
__device__ void block_sum2(double& a0, double& a1) {
  __shared__ double red[32][2];
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    a0 += __shfl_xor_sync(0xffffffffu, a0, off);
    a1 += __shfl_xor_sync(0xffffffffu, a1, off);
  }
  const int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) {
    red[w][0] = a0;
    red[w][1] = a1;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double s0 = 0.0, s1 = 0.0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) {
      s0 += red[k][0];
      s1 += red[k][1];
    }
    a0 = s0;
    a1 = s1;
  }
  __syncthreads();
}

// out[2 sg + {0,1}] = sums of the per-row dots over segment sg's block rows.
__global__ void seg_row_dots_kernel(const double* __restrict__ row_dots, const int* __restrict__ seg_rows, int nseg,
                                    double* __restrict__ out) {
  for (int sg = blockIdx.x; sg < nseg; sg += gridDim.x) {
    double a0 = 0.0, a1 = 0.0;
    for (int i = seg_rows[sg] + threadIdx.x; i < seg_rows[sg + 1]; i += blockDim.x) {
      a0 += row_dots[2 * i];
      a1 += row_dots[2 * i + 1];
    }
    block_sum2(a0, a1);
    if (threadIdx.x == 0) {
      out[2 * sg] = a0;
      out[2 * sg + 1] = a1;
    }
  }
}

// out[2 sg] = sum |x|^2 over segment sg's scalar rows (all ld lanes).
template <typename T>
__global__ void seg_sumsq_kernel(const T* __restrict__ x, const int64_t* __restrict__ seg_scal, int ld, int nseg,
                                 double* __restrict__ out) {
  for (int sg = blockIdx.x; sg < nseg; sg += gridDim.x) {
    double a0 = 0.0, a1 = 0.0;
    for (int64_t i = seg_scal[sg] * ld + threadIdx.x; i < seg_scal[sg + 1] * ld; i += blockDim.x)
      a0 += re_dot(x[i], x[i]);
    block_sum2(a0, a1);
    if (threadIdx.x == 0) {
      out[2 * sg] = a0;
      out[2 * sg + 1] = 0.0;
    }
  }
}

static int ensure_grid_scratch(const vbg_matrix* m) { return ensure_scratch(m, max_total_ctas()); }

template <typename T>
static int launch_sumsq(const vbg_matrix* m, const T* x, int64_t n, double* out, cudaStream_t s) {
  int grid = (int)std::min<int64_t>((n + kThreads - 1) / kThreads, (int64_t)sm_count() * 8);
  grid = std::max(grid, 1);
  sumsq_kernel<T><<<grid, kThreads, 0, s>>>(x, n, m->partials.as<double>(), m->counter.as<unsigned>(), out);
  VBG_CUDA(cudaGetLastError());
  return 0;
}

// Runs the autotuner for the forward applies of a Chebyshev recurrence on
// these buffers (before a graph capture, where it cannot run): one step
// Y = 2 A X - Xprev with its dots (per block row when row_dots is set).
template <typename T>
static int tune_recurrence(const vbg_matrix* m, bool f32, int R, int ld, const T* X, const T* Xprev, T* Y,
                           double* dots, double* row_dots, cudaStream_t s) {
  ApplyArgs a;
  int rc = prepare(m, false, R, ld, a, s);
  if (rc) return rc;
  if (R <= 1) {
    // the vector kernel's records and choice, before a graph capture
    if (!a.slot_meta || row_dots) return 0;
    a.X = X;
    a.Xprev = Xprev;
    a.Y = Y;
    a.alpha = 2.0;
    a.gamma = -1.0;
    a.n_scal = m->N;
    const int2* sr;
    const T* v = f32 ? reinterpret_cast<const T*>(m->vals32.as<float>()) : reinterpret_cast<const T*>(m->vals.p);
    return vec_kernel<T>(m, f32, a, v, s, true, &sr);
  }
  a.X = X;
  a.Xprev = Xprev;
  a.Y = Y;
  a.alpha = 2.0;
  a.gamma = -1.0;
  a.want_dots = 1;
  a.partials = m->partials.as<double>();
  a.counter = m->counter.as<unsigned>();
  a.dots_out = dots;
  a.row_dots = row_dots;
  const T* v = f32 ? reinterpret_cast<const T*>(m->vals32.as<float>()) : reinterpret_cast<const T*>(m->vals.p);
  int which = -1;
  return fwd_choice<T>(m, f32, a, v, s, true, &which);
}

// Enqueues the whole KPM recurrence on stream s.
template <typename T>
static int kpm_enqueue(const vbg_matrix* m, int R, int ld, const T* V0, int M, bool f32, int two_moment, T* B0,
                       T* B1, T* B2, double* dots, double* moments, cudaStream_t s) {
  int rc = launch_sumsq<T>(m, V0, m->N * (int64_t)ld, dots, s);
  if (rc) return rc;
  if (M >= 2) {
    ApplyArgs a;
    if ((rc = prepare(m, false, R, ld, a, s))) return rc;
    a.want_dots = 1;
    a.partials = m->partials.as<double>();
    a.counter = m->counter.as<unsigned>();
    // t_1 = A t_0
    a.X = V0;
    a.Y = B0;
    a.alpha = 1.0;
    a.dotw = V0;
    a.dots_out = dots + 2;
    if ((rc = launch_apply(m, false, f32, a, s))) return rc;
    T* bufs[3] = {B0, B1, B2};
    const T* prev = V0;
    const T* cur = B0;
    int nb = 1;
    const int steps = two_moment ? (M - 2) / 2 : M - 2;  // SpMMs after the first
    for (int n = 1; n <= steps; ++n) {
      T* next = bufs[nb];
      nb = (nb + 1) % 3;
      a.X = cur;
      a.Xprev = prev;
      a.Y = next;
      a.alpha = 2.0;
      a.gamma = -1.0;
      a.dotw = two_moment ? nullptr : V0;
      a.dots_out = dots + 2 * (n + 1);
      if ((rc = launch_apply(m, false, f32, a, s))) return rc;
      prev = cur;
      cur = next;
    }
  }
  kpm_finalize<<<1, 32, 0, s>>>(dots, M, two_moment, moments, 2, 1);
  VBG_CUDA(cudaGetLastError());
  return 0;
}

}  // namespace vbg

using namespace vbg;

extern "C" {

int vbg_set_option(const char* name, long long value) {
  VBG_CHECK(name, VBG_E_ARG, "null option name");
  if (std::strcmp(name, "apply.chain") == 0) {
    VBG_CHECK(value >= 0 && value <= 2, VBG_E_ARG, "apply.chain takes 0, 1 or 2");
    g_opt_chain.store((int)value);
    return 0;
  }
  if (std::strcmp(name, "apply.autotune") == 0) {
    g_opt_autotune.store(value != 0 ? 1 : 0);
    return 0;
  }
  if (std::strcmp(name, "apply.vec_lanes") == 0) {
    VBG_CHECK(value == 0 || value == 1 || value == 2 || value == 4 || value == 8, VBG_E_ARG,
              "apply.vec_lanes takes 0, 1, 2, 4 or 8");
    g_opt_vec_lanes.store((int)value);
    return 0;
  }
  if (std::strcmp(name, "apply.vec_kernel") == 0) {
    VBG_CHECK(value >= 0 && value <= 2, VBG_E_ARG, "apply.vec_kernel takes 0, 1 or 2");
    g_opt_vec_kernel.store((int)value);
    return 0;
  }
  return fail(VBG_E_ARG, std::string("unknown option '") + name + "'");
}

int vbg_get_option(const char* name, long long* value) {
  VBG_CHECK(name && value, VBG_E_ARG, "null argument");
  if (std::strcmp(name, "apply.chain") == 0) {
    *value = g_opt_chain.load();
    return 0;
  }
  if (std::strcmp(name, "apply.autotune") == 0) {
    *value = g_opt_autotune.load();
    return 0;
  }
  if (std::strcmp(name, "apply.vec_lanes") == 0) {
    *value = g_opt_vec_lanes.load();
    return 0;
  }
  if (std::strcmp(name, "apply.vec_kernel") == 0) {
    *value = g_opt_vec_kernel.load();
    return 0;
  }
  return fail(VBG_E_ARG, std::string("unknown option '") + name + "'");
}

int vbg_device_status(unsigned* status, int clear) {
  VBG_CHECK(status, VBG_E_ARG, "null argument");
  VBG_CUDA(cudaMemcpyFromSymbol(status, g_pipe_status, sizeof(unsigned)));
  if (clear) {
    const unsigned zero = 0;
    VBG_CUDA(cudaMemcpyToSymbol(g_pipe_status, &zero, sizeof(unsigned)));
  }
  return 0;
}

int vbg_spmv(const vbg_matrix* m, const void* x, void* y, void* stream) {
  ApplyArgs a;
  cudaStream_t s = as_stream(stream);
  int rc = prepare(m, false, 1, 1, a, s);
  if (rc) return rc;
  VBG_CHECK(x && y, VBG_E_ARG, "null vector");
  a.X = x;
  a.Y = y;
  return launch_apply(m, false, false, a, s);
}

int vbg_spmv_adjoint(const vbg_matrix* m, const void* x, void* y, void* stream) {
  ApplyArgs a;
  cudaStream_t s = as_stream(stream);
  int rc = prepare(m, true, 1, 1, a, s);
  if (rc) return rc;
  VBG_CHECK(x && y, VBG_E_ARG, "null vector");
  a.X = x;
  a.Y = y;
  return launch_apply(m, true, false, a, s);
}

int vbg_spmm(const vbg_matrix* m, int k, int ld, const void* X, void* Y, void* stream) {
  ApplyArgs a;
  cudaStream_t s = as_stream(stream);
  int rc = prepare(m, false, k, ld, a, s);
  if (rc) return rc;
  VBG_CHECK(X && Y, VBG_E_ARG, "null multivector");
  a.X = X;
  a.Y = Y;
  return launch_apply(m, false, false, a, s);
}

int vbg_apply_tile_rows(const vbg_matrix* m, int ld, int precision, int* rows) {
  VBG_CHECK(m && rows, VBG_E_ARG, "null argument");
  VBG_CHECK(precision == VBG_PREC_F64 || (precision == VBG_PREC_F32 && m->dtype == VBG_F64), VBG_E_ARG,
            "precision must be VBG_PREC_F64, or VBG_PREC_F32 for a real matrix");
  const int es = precision == VBG_PREC_F32 ? 4 : (int)elem_size(m->dtype);
  *rows = 0;
  auto it = m->tile_plans.find(std::make_tuple(ld * es, es, tile_cap(m, ld, es)));
  if (it != m->tile_plans.end()) *rows = it->second->rows;
  return 0;
}

int vbg_apply_kernel(const vbg_matrix* m, int ld, int precision, int* kernel) {
  VBG_CHECK(m && kernel, VBG_E_ARG, "null argument");
  VBG_CHECK(precision == VBG_PREC_F64 || (precision == VBG_PREC_F32 && m->dtype == VBG_F64), VBG_E_ARG,
            "precision must be VBG_PREC_F64, or VBG_PREC_F32 for a real matrix");
  ApplyArgs a;
  int rc = prepare(m, false, 1, ld, a, nullptr);
  if (rc) return rc;
  if (ld <= 1) {
    *kernel = VBG_KERNEL_VECTOR;
    if (a.slot_meta && srow_possible(m)) {
      const int forced = g_opt_vec_kernel.load();
      auto it = m->tuned.find(std::make_pair(1, precision == VBG_PREC_F32 ? 1 : 0));
      if (forced == 2 || (forced == 0 && (it != m->tuned.end() ? it->second != VBG_KERNEL_VECTOR
                                                              : (m->dtype == VBG_C128 && precision == VBG_PREC_F64))))
        *kernel = VBG_KERNEL_SCALAR_ROWS;
    }
    return 0;
  }
  // the autotuner's choice once it has made one
  if (g_opt_autotune.load() && g_opt_chain.load() == 2) {
    auto it = m->tuned.find(std::make_pair(ld, precision == VBG_PREC_F32 ? 1 : 0));
    if (it != m->tuned.end()) {
      *kernel = it->second;
      return 0;
    }
  }
  // buffers aligned as the library's own allocations are
  a.X = a.Y = reinterpret_cast<void*>(static_cast<uintptr_t>(256));
  TilePlan* tp = nullptr;
  ChainPlan* cp = nullptr;
  bool chain, tile, pipe;
  const bool chain_ok = chain_enabled(precision == VBG_PREC_F32 ? 4 : (int)elem_size(m->dtype));
  if (precision == VBG_PREC_F32) {
    chain = chain_ok && (chain_use<float>(m, a, nullptr, true, &cp) || chain_use<float, 1>(m, a, nullptr, true, &cp) ||
                         chain_use<float, 1, 2>(m, a, nullptr, true, &cp));
    tile = chain || tile_use<float>(m, false, a, nullptr, true, &tp) ||
           tile_use<float, 1>(m, false, a, nullptr, true, &tp) || tile_use<float, 1, 2>(m, false, a, nullptr, true, &tp);
    pipe = tile || pipe_use<float>(m, false, a, nullptr, true);
  } else if (m->dtype == VBG_C128) {
    chain = chain_ok && chain_use<cplx>(m, a, nullptr, true, &cp);
    tile = chain || tile_use<cplx>(m, false, a, nullptr, true, &tp);
    pipe = tile || pipe_use<cplx>(m, false, a, nullptr, true);
  } else {
    chain = chain_ok && (chain_use<double>(m, a, nullptr, true, &cp) || chain_use<double, 1, 2>(m, a, nullptr, true, &cp));
    tile = chain || tile_use<double>(m, false, a, nullptr, true, &tp) ||
           tile_use<double, 1, 2>(m, false, a, nullptr, true, &tp);
    pipe = tile || pipe_use<double>(m, false, a, nullptr, true);
  }
  *kernel = chain ? VBG_KERNEL_CHAIN : tile ? VBG_KERNEL_TILE : pipe ? VBG_KERNEL_PIPE : VBG_KERNEL_ROWS;
  return 0;
}

int vbg_spmm_adjoint(const vbg_matrix* m, int k, int ld, const void* X, void* Y, void* stream) {
  ApplyArgs a;
  cudaStream_t s = as_stream(stream);
  int rc = prepare(m, true, k, ld, a, s);
  if (rc) return rc;
  VBG_CHECK(X && Y, VBG_E_ARG, "null multivector");
  a.X = X;
  a.Y = Y;
  return launch_apply(m, true, false, a, s);
}

// The fused step of vbg_cheb_step / vbg_cheb_step_adjoint.
static int fused_step(const vbg_matrix* m, bool adj, int k, int ld, double alpha, double beta, double gamma,
                      const void* X, const void* Xprev, void* Y, const void* dot_with, double* dots, void* acc,
                      double cre, double cim, void* stream) {
  ApplyArgs a;
  cudaStream_t s = as_stream(stream);
  int rc = prepare(m, adj, k, ld, a, s);
  if (rc) return rc;
  VBG_CHECK(X && Y, VBG_E_ARG, "null multivector");
  VBG_CHECK(gamma == 0.0 || Xprev, VBG_E_ARG, "Xprev is required when gamma != 0");
  a.alpha = alpha;
  a.beta = beta;
  a.gamma = gamma;
  a.X = X;
  a.Xprev = Xprev;
  a.Y = Y;
  a.dotw = dot_with;
  a.acc = acc;
  a.cre = cre;
  a.cim = cim;
  if (dots) {
    if ((rc = ensure_grid_scratch(m))) return rc;
    a.want_dots = 1;
    a.partials = m->partials.as<double>();
    a.counter = m->counter.as<unsigned>();
    a.dots_out = dots;
  }
  return launch_apply(m, adj, false, a, s);
}

int vbg_cheb_step(const vbg_matrix* m, int k, int ld, double alpha, double beta, double gamma, const void* X,
                  const void* Xprev, void* Y, const void* dot_with, double* dots, void* acc, double cre, double cim,
                  void* stream) {
  return fused_step(m, false, k, ld, alpha, beta, gamma, X, Xprev, Y, dot_with, dots, acc, cre, cim, stream);
}

int vbg_cheb_step_adjoint(const vbg_matrix* m, int k, int ld, double alpha, double beta, double gamma, const void* X,
                          const void* Xprev, void* Y, const void* dot_with, double* dots, void* acc, double cre,
                          double cim, void* stream) {
  return fused_step(m, true, k, ld, alpha, beta, gamma, X, Xprev, Y, dot_with, dots, acc, cre, cim, stream);
}

int vbg_cheb_series(const vbg_matrix* m, int k, int ld, const void* V, int M, const double* coeffs, double scale,
                    double center, void* psi, int K, void* ckpt, void* stream) {
  VBG_CHECK(m && V && psi && coeffs, VBG_E_ARG, "null argument");
  VBG_CHECK(M >= 1 && k >= 1 && ld >= k && scale != 0.0, VBG_E_ARG, "invalid M / k / ld / scale");
  VBG_CHECK(K <= 0 || ckpt || M <= K, VBG_E_ARG, "checkpoint buffer required when K > 0");
  const int dtype = m->dtype;
  const size_t es = elem_size(dtype);
  const int64_t rows = m->N;
  const size_t bytes = (size_t)rows * (size_t)ld * es;
  cudaStream_t s = as_stream(stream);
  int rc;
  // psi = c_0 t_0
  VBG_CUDA(cudaMemsetAsync(psi, 0, bytes, s));
  if ((rc = vbg_mv_axpby(dtype, rows, k, ld, coeffs[0], coeffs[1], V, 0.0, 0.0, psi, stream))) return rc;
  if (M == 1) return 0;
  DevBuf buf[3] = {DevBuf(s), DevBuf(s), DevBuf(s)};
  for (auto& b : buf) {
    if ((rc = b.ensure(std::max<size_t>(bytes, 16)))) return rc;
    VBG_CUDA(cudaMemsetAsync(b.p, 0, bytes, s));  // pad lanes stay zero
  }
  const int n_ck = K > 0 ? (M - 1) / K : 0;
  if (n_ck > 0) VBG_CUDA(cudaMemsetAsync(ckpt, 0, (size_t)2 * n_ck * bytes, s));
  const void* t_prev = nullptr;
  const void* t = V;
  // t_n is written straight into its checkpoint slot when n = K, 2K, ...
  // (vector 2j) or n + 1 is (vector 2j + 1), else into a working vector
  // that holds neither t_{n-1} nor t_{n-2}
  auto slot = [&](int j, int w) { return static_cast<char*>(ckpt) + (size_t)(2 * j + w) * bytes; };
  for (int n = 1; n < M; ++n) {
    void* y = nullptr;
    if (K > 0 && n % K == 0)
      y = slot(n / K - 1, 0);
    else if (K > 0 && (n + 1) % K == 0 && n + 1 < M)
      y = slot((n + 1) / K - 1, 1);
    else
      for (auto& b : buf)
        if (b.p != t && b.p != t_prev) {
          y = b.p;
          break;
        }
    const bool first = n == 1;
    const double alpha = (first ? 1.0 : 2.0) / scale;
    const double beta = -(first ? 1.0 : 2.0) * center / scale;
    const double gamma = first ? 0.0 : -1.0;
    if ((rc = vbg_cheb_step(m, k, ld, alpha, beta, gamma, t, first ? nullptr : t_prev, y, nullptr, nullptr, psi,
                            coeffs[2 * n], coeffs[2 * n + 1], stream)))
      return rc;
    // K = 1: t_{n-1} sits in the previous pair's slot (or is V)
    if (K > 0 && n % K == 0 && t != slot(n / K - 1, 1))
      VBG_CUDA(cudaMemcpyAsync(slot(n / K - 1, 1), t, bytes, cudaMemcpyDeviceToDevice, s));
    t_prev = t;
    t = y;
  }
  return 0;
}

int vbg_kpm_moments(const vbg_matrix* m, int R, int ld, const void* V0, int M, int precision, int two_moment,
                    int use_graph, double* moments, void* stream) {
  VBG_CHECK(m && V0 && moments, VBG_E_ARG, "null argument");
  VBG_CHECK(m->dtype == VBG_F64, VBG_E_ARG, "KPM moments are defined for real symmetric matrices");
  VBG_CHECK(R >= 1 && ld >= R && M >= 1, VBG_E_ARG, "invalid R / ld / M");
  VBG_CHECK(precision == VBG_PREC_F64 || precision == VBG_PREC_F32, VBG_E_ARG, "unknown precision");
  VBG_CHECK(R == 1 ? true : (ld * 8) % 16 == 0, VBG_E_ARG, "ld must span a multiple of 16 bytes");
  cudaStream_t s = as_stream(stream);
  auto* mm = const_cast<vbg_matrix*>(m);
  int rc = ensure_grid_scratch(m);
  if (rc) return rc;
  const bool f32 = precision == VBG_PREC_F32;
  // FP32 multivectors use the reference's padding rule for 4-byte scalars.
  const int ldw = f32 ? (R == 1 ? 1 : ((R * 4 + 63) / 64) * 16) : ld;
  const size_t es = f32 ? 4 : 8;
  const size_t nbuf = f32 ? 4 : 3;
  const size_t buf_bytes = ((size_t)m->N * ldw * es + 255) / 256 * 256;
  const void* ws_before = mm->kpm_ws.p;
  const void* dots_before = mm->kpm_dots.p;
  if ((rc = mm->kpm_ws.ensure(std::max<size_t>(nbuf * buf_bytes, 256)))) return rc;
  const int nsteps = M + 2;
  if ((rc = mm->kpm_dots.ensure((size_t)nsteps * 2 * sizeof(double)))) return rc;
  // captured graphs hold raw workspace pointers
  if (mm->kpm_ws.p != ws_before || mm->kpm_dots.p != dots_before) mm->graphs.clear();
  char* base = mm->kpm_ws.as<char>();
  double* dots = mm->kpm_dots.as<double>();
  if (f32) {
    const int64_t tot = m->N * (int64_t)ldw;
    f64_to_f32_rows<<<std::max<int64_t>(1, std::min<int64_t>((tot + 255) / 256, sm_count() * 16)), 256, 0, s>>>(
        static_cast<const double*>(V0), m->N, ld, reinterpret_cast<float*>(base + 3 * buf_bytes), ldw);
    VBG_CUDA(cudaGetLastError());
    if ((rc = ensure_vals32(m, s))) return rc;
  }
  // the pipelined kernel's value layout must exist before a graph capture
  if (R > 1 && m->max_bs <= kPipeMaxBs && (f32 ? pipe_groups<float>(ldw) : pipe_groups<double>(ldw)) != 0) {
    if ((rc = ensure_kernel_layout(m, f32, s))) return rc;
    if ((rc = ensure_spans(m, pipe_span_cap(m), s))) return rc;
    if ((rc = tile_prepare(m, f32, ldw, s))) return rc;
  }
  // the kernel choice, before a graph capture freezes it
  if (f32)
    rc = tune_recurrence<float>(m, true, R, ldw, reinterpret_cast<const float*>(base + 3 * buf_bytes),
                                reinterpret_cast<const float*>(base + buf_bytes), reinterpret_cast<float*>(base),
                                dots + 2, nullptr, s);
  else
    rc = tune_recurrence<double>(m, false, R, ldw, static_cast<const double*>(V0),
                                 reinterpret_cast<const double*>(base + buf_bytes), reinterpret_cast<double*>(base),
                                 dots + 2, nullptr, s);
  if (rc) return rc;
  auto enqueue = [&](cudaStream_t st) -> int {
    if (f32)
      return kpm_enqueue<float>(m, R, ldw, reinterpret_cast<const float*>(base + 3 * buf_bytes), M, true, two_moment,
                                reinterpret_cast<float*>(base), reinterpret_cast<float*>(base + buf_bytes),
                                reinterpret_cast<float*>(base + 2 * buf_bytes), dots, moments, st);
    return kpm_enqueue<double>(m, R, ldw, static_cast<const double*>(V0), M, false, two_moment,
                               reinterpret_cast<double*>(base), reinterpret_cast<double*>(base + buf_bytes),
                               reinterpret_cast<double*>(base + 2 * buf_bytes), dots, moments, st);
  };
  if (!use_graph) return enqueue(s);

  auto key = std::make_tuple(R, ld, V0, M, precision, two_moment, moments);
  auto it = mm->graphs.find(key);
  if (it == mm->graphs.end()) {
    if (!mm->graph_stream) VBG_CUDA(cudaStreamCreateWithFlags(&mm->graph_stream, cudaStreamNonBlocking));
    auto ge = std::make_unique<GraphEntry>();
    VBG_CUDA(cudaStreamBeginCapture(mm->graph_stream, cudaStreamCaptureModeThreadLocal));
    rc = enqueue(mm->graph_stream);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(mm->graph_stream, &g);
    if (rc) {
      if (g) cudaGraphDestroy(g);
      return rc;
    }
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
    ge->graph = g;
    VBG_CUDA(cudaGraphInstantiate(&ge->exec, g, 0));
    it = mm->graphs.emplace(key, std::move(ge)).first;
  }
  VBG_CUDA(cudaGraphLaunch(it->second->exec, s));
  return 0;
}

int vbg_kpm_moments_host(const vbg_matrix* m, int R, const double* V0, int M, int precision, int two_moment,
                         double* moments, void* stream) {
  VBG_CHECK(m && V0 && moments, VBG_E_ARG, "null argument");
  VBG_CHECK(R >= 1 && M >= 1, VBG_E_ARG, "invalid R / M");
  cudaStream_t s = as_stream(stream);
  const int ld = R == 1 ? 1 : ((R * 8 + 63) / 64) * 8;
  DevBuf dv, dm;
  int rc;
  if ((rc = dv.ensure((size_t)m->N * ld * 8))) return rc;
  if ((rc = dm.ensure((size_t)M * 8))) return rc;
  if (ld != R) VBG_CUDA(cudaMemsetAsync(dv.p, 0, (size_t)m->N * ld * 8, s));
  VBG_CUDA(cudaMemcpy2DAsync(dv.p, (size_t)ld * 8, V0, (size_t)R * 8, (size_t)R * 8, m->N, cudaMemcpyHostToDevice, s));
  if ((rc = vbg_kpm_moments(m, R, ld, dv.p, M, precision, two_moment, 0, dm.as<double>(), s))) return rc;
  VBG_CUDA(cudaMemcpyAsync(moments, dm.p, (size_t)M * 8, cudaMemcpyDeviceToHost, s));
  VBG_CUDA(cudaStreamSynchronize(s));
  return 0;
}

}  // extern "C"

namespace vbg {

// Enqueues the batched recurrence: one block-diagonal matrix whose diagonal
// blocks (segments) are independent Hamiltonians; every apply writes per-row
// dots that a segmented reduction turns into per-segment dots.
template <typename T>
static int kpm_enqueue_batched(const vbg_matrix* m, int nseg, const int* seg_rows, const int64_t* seg_scal, int R,
                               int ld, const T* V0, int M, bool f32, int two_moment, T* B0, T* B1, T* B2,
                               double* row_dots, double* dots, double* moments, cudaStream_t s) {
  const int stride = 2 * nseg;
  const int sgrid = std::max(1, std::min(nseg, sm_count() * 4));
  seg_sumsq_kernel<T><<<sgrid, 256, 0, s>>>(V0, seg_scal, ld, nseg, dots);
  VBG_CUDA(cudaGetLastError());
  if (M >= 2) {
    ApplyArgs a;
    int rc;
    if ((rc = prepare(m, false, R, ld, a, s))) return rc;
    a.want_dots = 1;
    a.row_dots = row_dots;
    a.X = V0;
    a.Y = B0;
    a.alpha = 1.0;
    a.dotw = V0;
    if ((rc = launch_apply(m, false, f32, a, s))) return rc;
    seg_row_dots_kernel<<<sgrid, 256, 0, s>>>(row_dots, seg_rows, nseg, dots + stride);
    VBG_CUDA(cudaGetLastError());
    T* bufs[3] = {B0, B1, B2};
    const T* prev = V0;
    const T* cur = B0;
    int nb = 1;
    const int steps = two_moment ? (M - 2) / 2 : M - 2;
    for (int n = 1; n <= steps; ++n) {
      T* next = bufs[nb];
      nb = (nb + 1) % 3;
      a.X = cur;
      a.Xprev = prev;
      a.Y = next;
      a.alpha = 2.0;
      a.gamma = -1.0;
      a.dotw = two_moment ? nullptr : V0;
      if ((rc = launch_apply(m, false, f32, a, s))) return rc;
      seg_row_dots_kernel<<<sgrid, 256, 0, s>>>(row_dots, seg_rows, nseg, dots + (size_t)stride * (n + 1));
      VBG_CUDA(cudaGetLastError());
      prev = cur;
      cur = next;
    }
  }
  kpm_finalize<<<(nseg + 127) / 128, 128, 0, s>>>(dots, M, two_moment, moments, stride, nseg);
  VBG_CUDA(cudaGetLastError());
  return 0;
}

}  // namespace vbg

extern "C" {

int vbg_kpm_moments_batched(const vbg_matrix* m, int nseg, const int* seg_rows, int R, int ld, const void* V0, int M,
                            int precision, int two_moment, int use_graph, double* moments, void* stream) {
  VBG_CHECK(m && seg_rows && V0 && moments, VBG_E_ARG, "null argument");
  VBG_CHECK(m->dtype == VBG_F64, VBG_E_ARG, "KPM moments are defined for real symmetric matrices");
  VBG_CHECK(nseg >= 1 && R >= 2 && ld >= R && M >= 1, VBG_E_ARG,
            "invalid nseg / R / ld / M (batched moments need a multivector, R >= 2)");
  VBG_CHECK((ld * 8) % 16 == 0, VBG_E_ARG, "ld must span a multiple of 16 bytes");
  VBG_CHECK(precision == VBG_PREC_F64 || precision == VBG_PREC_F32, VBG_E_ARG, "unknown precision");
  VBG_CHECK(seg_rows[0] == 0 && seg_rows[nseg] == m->n, VBG_E_ARG, "segments must cover the block rows");
  for (int i = 0; i < nseg; ++i) VBG_CHECK(seg_rows[i + 1] >= seg_rows[i], VBG_E_ARG, "segments not monotone");
  cudaStream_t s = as_stream(stream);
  auto* mm = const_cast<vbg_matrix*>(m);
  int rc;
  // segment tables (device), rebuilt when the layout changes
  std::vector<int> segv(seg_rows, seg_rows + nseg + 1);
  if (segv != mm->kpm_seg_host) {
    std::vector<int64_t> scal(nseg + 1);
    for (int i = 0; i <= nseg; ++i) scal[i] = m->h_scal_off[seg_rows[i]];
    if ((rc = mm->kpm_seg.ensure((nseg + 1) * sizeof(int)))) return rc;
    if ((rc = mm->kpm_segscal.ensure((nseg + 1) * sizeof(int64_t)))) return rc;
    VBG_CUDA(cudaMemcpyAsync(mm->kpm_seg.p, segv.data(), (nseg + 1) * sizeof(int), cudaMemcpyHostToDevice, s));
    VBG_CUDA(cudaMemcpyAsync(mm->kpm_segscal.p, scal.data(), (nseg + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, s));
    VBG_CUDA(cudaStreamSynchronize(s));
    mm->kpm_seg_host = segv;
    mm->graphs.clear();
  }
  const bool f32 = precision == VBG_PREC_F32;
  // FP32 multivectors use the reference's padding rule for 4-byte scalars
  // (16 columns stay 16: the tiled applies take them with two lane groups)
  const int ldw = f32 ? ((R * 4 + 63) / 64) * 16 : ld;
  const size_t es = f32 ? 4 : 8;
  const size_t nbuf = f32 ? 4 : 3;
  const size_t buf_bytes = ((size_t)m->N * ldw * es + 255) / 256 * 256;
  const void* ws_before = mm->kpm_ws.p;
  const void* dots_before = mm->kpm_dots.p;
  const void* rd_before = mm->kpm_rowdots.p;
  if ((rc = mm->kpm_ws.ensure(std::max<size_t>(nbuf * buf_bytes, 256)))) return rc;
  if ((rc = mm->kpm_dots.ensure((size_t)(M + 2) * 2 * nseg * sizeof(double)))) return rc;
  if ((rc = mm->kpm_rowdots.ensure((size_t)std::max(m->n, 1) * 2 * sizeof(double)))) return rc;
  if (mm->kpm_ws.p != ws_before || mm->kpm_dots.p != dots_before || mm->kpm_rowdots.p != rd_before)
    mm->graphs.clear();
  char* base = mm->kpm_ws.as<char>();
  double* dots = mm->kpm_dots.as<double>();
  double* row_dots = mm->kpm_rowdots.as<double>();
  if (f32) {
    const int64_t tot = m->N * (int64_t)ldw;
    f64_to_f32_rows<<<std::max<int64_t>(1, std::min<int64_t>((tot + 255) / 256, sm_count() * 16)), 256, 0, s>>>(
        static_cast<const double*>(V0), m->N, ld, reinterpret_cast<float*>(base + 3 * buf_bytes), ldw);
    VBG_CUDA(cudaGetLastError());
    if ((rc = ensure_vals32(m, s))) return rc;
  }
  if (m->max_bs <= kPipeMaxBs && (f32 ? pipe_groups<float>(ldw) : pipe_groups<double>(ldw)) != 0) {
    if ((rc = ensure_kernel_layout(m, f32, s))) return rc;
    if ((rc = ensure_spans(m, pipe_span_cap(m), s))) return rc;
    if ((rc = tile_prepare(m, f32, ldw, s))) return rc;
  }
  if ((rc = ensure_grid_scratch(m))) return rc;
  if (f32)
    rc = tune_recurrence<float>(m, true, R, ldw, reinterpret_cast<const float*>(base + 3 * buf_bytes),
                                reinterpret_cast<const float*>(base + buf_bytes), reinterpret_cast<float*>(base),
                                dots, row_dots, s);
  else
    rc = tune_recurrence<double>(m, false, R, ldw, static_cast<const double*>(V0),
                                 reinterpret_cast<const double*>(base + buf_bytes), reinterpret_cast<double*>(base),
                                 dots, row_dots, s);
  if (rc) return rc;
  const int* sr = mm->kpm_seg.as<int>();
  const int64_t* ss = mm->kpm_segscal.as<int64_t>();
  auto enqueue = [&](cudaStream_t st) -> int {
    if (f32)
      return kpm_enqueue_batched<float>(m, nseg, sr, ss, R, ldw, reinterpret_cast<const float*>(base + 3 * buf_bytes),
                                        M, true, two_moment, reinterpret_cast<float*>(base),
                                        reinterpret_cast<float*>(base + buf_bytes),
                                        reinterpret_cast<float*>(base + 2 * buf_bytes), row_dots, dots, moments, st);
    return kpm_enqueue_batched<double>(m, nseg, sr, ss, R, ldw, static_cast<const double*>(V0), M, false, two_moment,
                                       reinterpret_cast<double*>(base), reinterpret_cast<double*>(base + buf_bytes),
                                       reinterpret_cast<double*>(base + 2 * buf_bytes), row_dots, dots, moments, st);
  };
  if (!use_graph) return enqueue(s);
  auto key = std::make_tuple(R, ld, V0, M, precision, two_moment + 2, moments);
  auto it = mm->graphs.find(key);
  if (it == mm->graphs.end()) {
    if (!mm->graph_stream) VBG_CUDA(cudaStreamCreateWithFlags(&mm->graph_stream, cudaStreamNonBlocking));
    auto ge = std::make_unique<GraphEntry>();
    VBG_CUDA(cudaStreamBeginCapture(mm->graph_stream, cudaStreamCaptureModeThreadLocal));
    rc = enqueue(mm->graph_stream);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(mm->graph_stream, &g);
    if (rc) {
      if (g) cudaGraphDestroy(g);
      return rc;
    }
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
    ge->graph = g;
    VBG_CUDA(cudaGraphInstantiate(&ge->exec, g, 0));
    it = mm->graphs.emplace(key, std::move(ge)).first;
  }
  VBG_CUDA(cudaGraphLaunch(it->second->exec, s));
  return 0;
}

int vbg_spmv_host(const vbg_matrix* m, const void* x, void* y, void* stream) {
  VBG_CHECK(m && x && y, VBG_E_ARG, "null argument");
  cudaStream_t s = as_stream(stream);
  const size_t bytes = (size_t)m->N * elem_size(m->dtype);
  DevBuf dx, dy;
  int rc;
  if ((rc = dx.ensure(bytes))) return rc;
  if ((rc = dy.ensure(bytes))) return rc;
  VBG_CUDA(cudaMemcpyAsync(dx.p, x, bytes, cudaMemcpyHostToDevice, s));
  if ((rc = vbg_spmv(m, dx.p, dy.p, s))) return rc;
  VBG_CUDA(cudaMemcpyAsync(y, dy.p, bytes, cudaMemcpyDeviceToHost, s));
  VBG_CUDA(cudaStreamSynchronize(s));
  return 0;
}

int vbg_spmm_host(const vbg_matrix* m, int k, const void* X, void* Y, void* stream) {
  VBG_CHECK(m && X && Y && k >= 1, VBG_E_ARG, "invalid argument");
  cudaStream_t s = as_stream(stream);
  const size_t es = elem_size(m->dtype);
  const int ld = k == 1 ? 1 : (int)(((k * es + 63) / 64) * 64 / es);
  const size_t bytes = (size_t)m->N * ld * es;
  DevBuf dx, dy;
  int rc;
  if ((rc = dx.ensure(bytes))) return rc;
  if ((rc = dy.ensure(bytes))) return rc;
  if (ld != k) VBG_CUDA(cudaMemsetAsync(dx.p, 0, bytes, s));
  VBG_CUDA(cudaMemcpy2DAsync(dx.p, ld * es, X, k * es, k * es, m->N, cudaMemcpyHostToDevice, s));
  if ((rc = vbg_spmm(m, k, ld, dx.p, dy.p, s))) return rc;
  VBG_CUDA(cudaMemcpy2DAsync(Y, k * es, dy.p, ld * es, k * es, m->N, cudaMemcpyDeviceToHost, s));
  VBG_CUDA(cudaStreamSynchronize(s));
  return 0;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free variant of the fused Chebyshev step.
//
// vbg_cheb_step keeps its per-CTA dot-product partials in scratch that the
// library allocates (cudaMalloc) on first use.  Some callers cannot allow
// any device allocation inside the library call: code that owns the whole
// device memory budget through its own pool or arena, or that runs where an
// allocation would synchronise the device at a point it must not.  For them
// vbg_cheb_step_noalloc takes that scratch from the file-scope array below
// instead.  The array is part of the library image: every GPU that loads the
// library holds it (64 KiB + 256 bytes) until the process exits.
namespace vbg {

// Per-CTA partial sums (two doubles each) for at most this many CTAs, then the
// grid-reduction counter.
constexpr int kNoAllocMaxCtas = 4096;
static __device__ __align__(256) double g_noalloc_scratch[2 * kNoAllocMaxCtas + 32];

// Device address of g_noalloc_scratch per device, looked up once per device.
static int noalloc_scratch(double** out) {
  static std::mutex mu;
  static std::map<int, double*> addr;
  int dev = 0;
  VBG_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(mu);
  auto it = addr.find(dev);
  if (it == addr.end()) {
    void* p = nullptr;
    VBG_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    it = addr.emplace(dev, static_cast<double*>(p)).first;
  }
  *out = it->second;
  return 0;
}

}  // namespace vbg

extern "C" int vbg_cheb_step_noalloc(const vbg_matrix* m, int k, int ld, double alpha, double beta, double gamma,
                                     const void* X, const void* Xprev, void* Y, const void* dot_with, double* dots,
                                     void* acc, double cre, double cim, void* stream) {
  ApplyArgs a;
  cudaStream_t s = as_stream(stream);
  int rc = prepare(m, false, k, ld, a, s);
  if (rc) return rc;
  VBG_CHECK(X && Y, VBG_E_ARG, "null multivector");
  VBG_CHECK(dots, VBG_E_ARG, "vbg_cheb_step_noalloc: dots is required (use vbg_cheb_step without dots)");
  VBG_CHECK(gamma == 0.0 || Xprev, VBG_E_ARG, "Xprev is required when gamma != 0");
  a.alpha = alpha;
  a.beta = beta;
  a.gamma = gamma;
  a.X = X;
  a.Xprev = Xprev;
  a.Y = Y;
  a.dotw = dot_with;
  a.acc = acc;
  a.cre = cre;
  a.cim = cim;
  double* scratch = nullptr;
  if ((rc = noalloc_scratch(&scratch))) return rc;
  unsigned* counter = reinterpret_cast<unsigned*>(scratch + 2 * kNoAllocMaxCtas);
  // the counter must start at zero; the previous call's value is not trusted
  VBG_CUDA(cudaMemsetAsync(counter, 0, sizeof(unsigned), s));
  a.want_dots = 1;
  a.partials = scratch;
  a.counter = counter;
  a.dots_out = dots;
  // the launcher checks the CTAs it actually starts against this room and
  // rejects the call (VBG_E_ARG) before any launch that would not fit
  a.max_ctas = kNoAllocMaxCtas;
  const int rc2 = launch_apply(m, false, false, a, s, false);
  if (rc2) set_error(std::string("vbg_cheb_step_noalloc: ") + vbg_last_error());
  return rc2;
}
