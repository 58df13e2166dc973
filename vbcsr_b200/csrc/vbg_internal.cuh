// Internal definitions shared by the vbcsr_b200 CUDA translation units.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <map>
#include <memory>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/vbcsr_b200.h"

namespace vbg {

// ------------------------------------------------------------- errors
void set_error(const std::string& msg);
int fail(int code, const std::string& msg);
int cuda_fail(cudaError_t e, const char* what);

#define VBG_CUDA(call)                                  \
  do {                                                  \
    cudaError_t e_ = (call);                            \
    if (e_ != cudaSuccess) return ::vbg::cuda_fail(e_, #call); \
  } while (0)

#define VBG_CHECK(cond, code, msg)                      \
  do {                                                  \
    if (!(cond)) return ::vbg::fail((code), (msg));     \
  } while (0)

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

// ------------------------------------------------------------- scalars
struct cplx {
  double re, im;
};

__host__ __device__ inline cplx operator+(cplx a, cplx b) { return {a.re + b.re, a.im + b.im}; }
__host__ __device__ inline cplx operator-(cplx a, cplx b) { return {a.re - b.re, a.im - b.im}; }

// Fused multiply-add helpers with one entry point per scalar type.
__device__ __forceinline__ double fma_s(double a, double x, double acc) { return fma(a, x, acc); }
__device__ __forceinline__ float fma_s(float a, float x, float acc) { return fmaf(a, x, acc); }
__device__ __forceinline__ cplx fma_s(cplx a, cplx x, cplx acc) {
  acc.re = fma(a.re, x.re, acc.re);
  acc.re = fma(-a.im, x.im, acc.re);
  acc.im = fma(a.re, x.im, acc.im);
  acc.im = fma(a.im, x.re, acc.im);
  return acc;
}
__device__ __forceinline__ double conj_s(double a) { return a; }
__device__ __forceinline__ float conj_s(float a) { return a; }
__device__ __forceinline__ cplx conj_s(cplx a) { return {a.re, -a.im}; }
template <typename T> __device__ __forceinline__ T zero_s();
template <> __device__ __forceinline__ double zero_s<double>() { return 0.0; }
template <> __device__ __forceinline__ float zero_s<float>() { return 0.0f; }
template <> __device__ __forceinline__ cplx zero_s<cplx>() { return {0.0, 0.0}; }
// Real part of conj(a) * b, in double.
__device__ __forceinline__ double re_dot(double a, double b) { return a * b; }
__device__ __forceinline__ double re_dot(float a, float b) { return (double)a * (double)b; }
__device__ __forceinline__ double re_dot(cplx a, cplx b) { return fma(a.re, b.re, a.im * b.im); }
// scale by a real double
__device__ __forceinline__ double scal_r(double s, double a) { return s * a; }
__device__ __forceinline__ float scal_r(double s, float a) { return (float)s * a; }
__device__ __forceinline__ cplx scal_r(double s, cplx a) { return {s * a.re, s * a.im}; }
// a*x + b for a real scale a
__device__ __forceinline__ double axpy_r(double a, double x, double b) { return fma(a, x, b); }
__device__ __forceinline__ float axpy_r(double a, float x, float b) { return fmaf((float)a, x, b); }
__device__ __forceinline__ cplx axpy_r(double a, cplx x, cplx b) { return {fma(a, x.re, b.re), fma(a, x.im, b.im)}; }
// complex-coefficient multiply-add c*x + b (imag ignored for real types)
__device__ __forceinline__ double cmad(double cr, double ci, double x, double b) { return fma(cr, x, b); }
__device__ __forceinline__ float cmad(double cr, double ci, float x, float b) { return fmaf((float)cr, x, b); }
__device__ __forceinline__ cplx cmad(double cr, double ci, cplx x, cplx b) {
  return {fma(cr, x.re, fma(-ci, x.im, b.re)), fma(cr, x.im, fma(ci, x.re, b.im))};
}

inline size_t elem_size(int dtype) { return dtype == VBG_C128 ? 16 : 8; }

// ------------------------------------------------------------- device buffer
// Device memory of the library (vbg_struct.cu).  Buffers of at least
// kCacheMinBytes come from a cache of cudaMalloc blocks per device (sizes
// rounded to powers of two from 32 MiB up), smaller ones from a
// stream-ordered pool per device.  Operations that build a new structure
// (SpGEMM, axpby on a union pattern, the block filter) allocate and release
// hundreds of MB per call; both keep that memory mapped between calls.  Two
// disciplines:
//   owned  (default constructor: matrix members, caches) -- released like
//          cudaFree: the device is synchronised first, so no kernel on any
//          stream can still use the memory when it is handed out again;
//          allocated on the stream given to ensure(n, s), or, without one,
//          on the legacy stream and waited for;
//   local  (DevBuf(stream): temporaries of one operation) -- allocated on
//          that stream and used on it only; released in stream order (pool)
//          or, for the cache, once an event recorded on that stream at the
//          release has completed.
// Neither kind may be allocated or released inside a stream capture.
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  cudaStream_t st = nullptr;  // local buffers: the stream of the operation
  bool local = false;
  bool cached = false;        // p came from the block cache (else the pool)
  DevBuf() = default;
  explicit DevBuf(cudaStream_t s) : st(s), local(true) {}
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { release(); }
  void release();
  // Release after the caller has synchronised the device (owned buffers).
  void release_synced();
  // Grows (never shrinks) to at least n bytes; contents are not preserved.
  int ensure(size_t n, cudaStream_t s);
  int ensure(size_t n) { return ensure(n, st); }
  template <typename T> T* as() const { return static_cast<T*>(p); }
};
// Page-locked host buffer kept for reuse (grows by half again, at least
// 1 MiB): device <-> host copies of per-row tables without pageable staging.
struct HostBuf {
  void* p = nullptr;
  size_t bytes = 0;
  HostBuf() = default;
  HostBuf(const HostBuf&) = delete;
  HostBuf& operator=(const HostBuf&) = delete;
  ~HostBuf() {
    if (p) cudaFreeHost(p);
  }
  int ensure(size_t n) {
    if (n <= bytes && p) return 0;
    if (p) cudaFreeHost(p);
    p = nullptr;
    bytes = 0;
    const size_t want = n + n / 2 > ((size_t)1 << 20) ? n + n / 2 : ((size_t)1 << 20);
    cudaError_t e = cudaHostAlloc(&p, want, cudaHostAllocDefault);
    if (e != cudaSuccess) {
      p = nullptr;
      (void)cudaGetLastError();
      return fail(VBG_E_NOMEM, "page-locked host allocation of " + std::to_string(want) + " bytes failed");
    }
    bytes = want;
    return 0;
  }
  template <typename T> T* as() const { return static_cast<T*>(p); }
};
// Exchanges the memory of two buffers (with its origin); each keeps its
// discipline.
inline void swap_mem(DevBuf& a, DevBuf& b) {
  std::swap(a.p, b.p);
  std::swap(a.bytes, b.bytes);
  std::swap(a.cached, b.cached);
}
// Returns the released, still mapped memory of the current device (block
// cache and pool) to the driver.
int trim_pool();
// Maps `bytes` into the current device's pool (and keeps them there).
int reserve_pool(size_t bytes);

// Row tiles of the tiled multivector apply: consecutive block rows whose X
// rows (the union over the tile's blocks: a few contiguous ranges) and
// kernel-layout values are staged in shared memory together.
struct TilePlan {
  int rows = 0;       // block rows per tile (= warps of the CTA)
  int ntiles = 0;
  int xcap = 0;       // staged X rows of the largest tile
  int owncap = 0;     // scalar rows of the largest tile
  int64_t vcap = 0;   // value scalars of the largest tile
  int qcap = 0;       // staged q-list bytes of the largest tile
  int grid = 0, smem = 0;
  // four int4 per tile: {first block row, end block row, first range, end
  // range}, {first value offset (two halves), value bytes, X bytes}, {shared
  // row of the first own X row, own scalar rows, first own scalar row, 0},
  // {first q-list entry staged, q-list bytes, 0, 0}
  DevBuf tiles;
  DevBuf ranges;      // int4 {first X row, X rows, first shared-memory row, 0}
  // The q-list: per block row, the shared-memory row of every X row its
  // blocks read, in slot order and column order within a block (uint16;
  // each row's list starts at a multiple of 4 entries).
  DevBuf qidx;
  // per block row: {its first q-list entry from the tile's first staged
  // entry, its q-list length, its first value from the tile's first value
  // (scalars, kernel layout), its block size}
  DevBuf rowinfo;
  // the kernel's work queue: {tiles claimed beyond the first wave, CTAs
  // done}; zero between launches (the last CTA of a launch resets it), so
  // launches with one plan must not overlap
  DevBuf queue;
};

// Row tiles of the chained tiled apply (vbg_chain.cuh): tiles in the order
// each persistent CTA processes them, with the X rows each tile has to load
// into the CTA's X cache (rows staged for earlier tiles of the same CTA are
// reused in place).
struct ChainPlan {
  int rows = 0;          // block rows per tile (= consumer warps of the CTA)
  int ntiles = 0;
  int nctas = 0;
  int cap_rows = 0;      // X rows the shared-memory cache holds
  int64_t vcap = 0;      // value scalars of the largest tile
  int qcap = 0;          // staged q-list bytes of the largest tile
  int stride = 0;        // tiles between consecutive tiles of a chain (0: natural order)
  int smem = 0;
  int64_t staged_rows = 0;  // X rows loaded per apply (all tiles), for reports
  // three int4 per tile in processing order: {first block row, end block
  // row, first load, end load}, {value offset (two halves), value bytes,
  // cache row of the tile's first own scalar row}, {first q-list entry
  // staged, q-list bytes, 0, 0}
  DevBuf tiles;
  DevBuf loads;          // int4 {first X row, X rows, first cache row, 0}
  DevBuf cta_ptr;        // nctas + 1 tile ranges (processing order)
  DevBuf qidx, rowinfo;  // as TilePlan's, in cache rows
};

// CUDA-graph cache entry for a replayable recurrence.
struct GraphEntry {
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  ~GraphEntry() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
  }
};

}  // namespace vbg

// The opaque handle behind the C ABI.
struct vbg_matrix {
  int dtype = VBG_F64;
  int device = 0;
  int n = 0;            // block rows == block columns
  int64_t nnzb = 0;     // stored blocks
  int64_t nnz = 0;      // stored scalars
  int64_t N = 0;        // scalar rows
  int kind = VBG_KIND_VBCSR;
  int max_bs = 0, min_bs = 0;

  // host copies of the structure.  h_bsz and h_scal_off are always
  // current; h_row_ptr, h_col_ind and h_blk_off only while host_struct is set
  // (a structure built on the device is read back on first host use:
  // ensure_host_structure)
  std::vector<int> h_row_ptr, h_col_ind, h_bsz;
  std::vector<int64_t> h_blk_off, h_scal_off;
  bool host_struct = true;
  // some block row holds a block column more than once
  bool dup_cols = false;

  // rows grouped by block size: row_perm[w0, w1) all have block size r
  struct ClassSeg {
    int r, w0, w1;
  };
  std::vector<ClassSeg> class_segs;

  // device structure
  vbg::DevBuf row_ptr, col_ind, bsz, scal_off, blk_off, diag_slot, row_perm;
  // per slot: {first scalar row of the block column, rows << 8 | cols}
  vbg::DevBuf slot_meta;
  // per scalar row, built lazily for the scalar-row vector apply: {first
  // slot of its block row, slot count << 8 | row inside the block}
  vbg::DevBuf srow;
  bool srow_valid = false;
  // the same for the adjoint over the column view, built lazily: per scalar
  // column {first column-view entry, count << 8 | column inside the block},
  // per column-view entry {first X row of its block row, rows << 8 | cols}
  // and its value offset
  vbg::DevBuf scol, csc_meta, csc_boff;
  bool scol_valid = false;
  // device values (FP64 / C128) and the lazily built FP32 shadow
  vbg::DevBuf vals, vals32;
  bool vals32_valid = false;
  // Kernel layout of the values for the pipelined multivector apply, built
  // lazily (blocks of at most 8 x 8 only): each block stored column by
  // column, every column padded to 16 bytes of scalars (kernel_layout_rows),
  // so a block is 16-byte aligned and its columns load as 16-byte vectors.
  // koff* are the per-slot offsets (nnzb + 1 entries) of the value type and
  // of the FP32 shadow.
  vbg::DevBuf valsK, valsK32, koff, koff32;
  int64_t koff_total = 0, koff32_total = 0;
  bool valsK_valid = false, valsK32_valid = false, koff_valid = false;
  // Spans of the pipelined apply: runs of consecutive slots of one block row
  // whose block columns are consecutive (their X rows and kernel-layout
  // values are contiguous), at most span_cap X rows each.  spans[i] =
  // {first X row, X rows | block rows << 8, kernel-layout value offset (two
  // halves)}; span_koff32 holds the FP32 layout's offsets; row_sptr gives
  // each block row's spans (n + 1 entries).
  vbg::DevBuf spans, span_koff32, row_sptr;
  int span_cap = 0;
  int64_t nspans = 0;
  std::vector<int> h_span_x, h_row_sptr;  // host copies: first X row of each span, row_sptr
  std::vector<unsigned char> h_span_w;    // and its X rows
  // Row tiles of the tiled multivector apply (vbg_tile.cuh), one plan per
  // (X row bytes, value scalar size, tile height cap), built lazily; the cap
  // in use per (leading dimension, value scalar size) is the autotuner's
  // (kTileRowsMax until it has run).
  std::map<std::tuple<int, int, int>, std::unique_ptr<vbg::TilePlan>> tile_plans;
  std::map<std::pair<int, int>, int> tile_rows_cap;
  // and whether its tiled kernel takes tiles from the work queue (1) or in
  // a fixed stride (0, the default)
  std::map<std::pair<int, int>, int> tile_queue;
  // Chained row tiles (vbg_chain.cuh), per (X row bytes, value scalar size).
  std::map<std::pair<int, int>, std::unique_ptr<vbg::ChainPlan>> chain_plans;
  // The autotuner's choice of forward multivector kernel (VBG_KERNEL_*) per
  // (leading dimension, FP32 values).
  std::map<std::pair<int, int>, int> tuned;
  // adjoint (column-major) view, built lazily
  vbg::DevBuf csc_ptr, csc_slot, csc_row, csc_perm;
  bool csc_valid = false;

  // scratch for fused reductions: one partial pair per CTA + a done counter
  vbg::DevBuf partials, counter;
  // KPM workspace and graph cache
  vbg::DevBuf kpm_ws, kpm_dots;
  // batched KPM: per-row dots, segment boundaries (block rows, scalar rows)
  vbg::DevBuf kpm_rowdots, kpm_seg, kpm_segscal;
  std::vector<int> kpm_seg_host;
  std::map<std::tuple<int, int, const void*, int, int, int, double*>, std::unique_ptr<vbg::GraphEntry>> graphs;
  cudaStream_t graph_stream = nullptr;

  void invalidate_values() {
    vals32_valid = false;
    valsK_valid = valsK32_valid = false;
    graphs.clear();
  }
  void invalidate_structure() {
    csc_valid = false;
    srow_valid = false;
    scol_valid = false;
    koff_valid = false;
    span_cap = 0;
    tile_plans.clear();
    tile_rows_cap.clear();
    tile_queue.clear();
    chain_plans.clear();
    tuned.clear();
    invalidate_values();
  }
  ~vbg_matrix() {
    graphs.clear();
    if (graph_stream) cudaStreamDestroy(graph_stream);
    // one device synchronisation for all owned buffers (each would otherwise
    // synchronise on its own release)
    cudaDeviceSynchronize();
    for (vbg::DevBuf* b : {&row_ptr, &col_ind, &bsz, &scal_off, &blk_off, &diag_slot, &row_perm, &slot_meta, &srow, &scol, &csc_meta, &csc_boff, &vals,
                           &vals32, &valsK, &valsK32, &koff, &koff32, &spans, &span_koff32, &row_sptr, &csc_ptr,
                           &csc_slot, &csc_row, &csc_perm, &partials, &counter, &kpm_ws, &kpm_dots, &kpm_rowdots,
                           &kpm_seg, &kpm_segscal})
      b->release_synced();
  }
};

namespace vbg {
// Structure helpers shared between translation units (vbg_matrix.cu).
int build_structure(vbg_matrix* m, int n, const int* bsz, const int* row_ptr, const int* col_ind,
                    std::vector<int64_t>* sort_perm_out);
int upload_structure(vbg_matrix* m, cudaStream_t s);
int device_slot_structure(vbg_matrix* m, cudaStream_t s);
int ensure_vals32(const vbg_matrix* m, cudaStream_t s);
// Rows of one block column in the kernel layout: r rounded up to a whole
// 16-byte vector of scalars of `es` bytes.
__host__ __device__ constexpr inline int kernel_layout_rows(int r, int es) {
  const int v = es >= 16 ? 1 : 16 / es;
  return (r + v - 1) / v * v;
}
// Builds (once per value change) the kernel layout of the values: FP64/C128
// (f32 = false) or the FP32 shadow (f32 = true).  Requires max_bs <= 8.
int ensure_kernel_layout(const vbg_matrix* m, bool f32, cudaStream_t s);
// Builds (once per structure and cap) the spans of the pipelined apply.
int ensure_spans(const vbg_matrix* m, int cap, cudaStream_t s);
int ensure_csc(const vbg_matrix* m, cudaStream_t s);
// Builds the column view (csc_ptr / csc_slot / csc_row / csc_perm) on the device.
int build_csc_dev(const vbg_matrix* m, cudaStream_t s);
// Device-side structure construction (vbg_struct.cu): exclusive prefix sum of
// n ints; a fresh matrix taking the device pattern (d_rp, d_ci; nnzb slots)
// with the block sizes of `like`; compaction of a matrix to its slots with
// keep[slot] != 0.
int exclusive_sum_int(const int* in, int* out, int64_t n, cudaStream_t s);
// Reads the device structure back into h_row_ptr / h_col_ind / h_blk_off
// when they are not current (synchronises s).
int ensure_host_structure(const vbg_matrix* m, cudaStream_t s);
int adopt_device_structure(vbg_matrix* m, const vbg_matrix* like, DevBuf& d_rp, DevBuf& d_ci, int64_t nnzb,
                           cudaStream_t s);
int compact_by_mask_dev(vbg_matrix* m, const unsigned char* keep, cudaStream_t s);
// Replaces an upper-block-triangle matrix U by U + strict_lower(U^H) with
// Hermitized diagonal blocks (vbg_algebra.cu).
int complete_hermitian_dev(vbg_matrix* U, cudaStream_t s);
int ensure_scratch(const vbg_matrix* m, int grid);
// Launch properties (SM count, occupancy, kernel attributes) are cached per
// device, indexed by the current device (ids >= kMaxDevices share the last
// slot, which only costs a re-query).
constexpr int kMaxDevices = 64;
int current_device();
int sm_count();
}  // namespace vbg
