// Device-side construction of a matrix structure: the result patterns of
// SpGEMM and of the block filter are produced on the device, so their slot
// offsets, gather metadata and diagonal slots are computed there too, and
// the host mirrors (row pointers, column lists, slot offsets) are read back
// once through a pinned staging buffer.  The alternative -- sending the
// pattern to the host and rebuilding everything there -- dominated the cost
// of a thresholded SpGEMM.
#include <algorithm>
#include <cstring>
#include <map>
#include <mutex>
#include <vector>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include "vbg_internal.cuh"

namespace vbg {

void move_into(vbg_matrix* dst, vbg_matrix* src);

// ------------------------------------------------------------- device pool
// Buffers below kCacheMinBytes: one stream-ordered pool per device, created
// on first use and kept for the life of the process.  Released memory stays
// mapped up to the release threshold (an eighth of the device memory); above
// it the pool returns memory to the driver at synchronisation points.
static std::mutex g_pool_mu;
constexpr size_t kPoolRoundBytes = (size_t)32 << 20;
static std::map<int, cudaMemPool_t> g_pools;

static int device_pool(cudaMemPool_t* out) {
  int dev = 0;
  VBG_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(g_pool_mu);
  auto it = g_pools.find(dev);
  if (it == g_pools.end()) {
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.handleTypes = cudaMemHandleTypeNone;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t pool = nullptr;
    VBG_CUDA(cudaMemPoolCreate(&pool, &props));
    size_t free_b = 0, total_b = 0;
    VBG_CUDA(cudaMemGetInfo(&free_b, &total_b));
    uint64_t thr = total_b / 8;
    VBG_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr));
    it = g_pools.emplace(dev, pool).first;
  }
  *out = it->second;
  return 0;
}

// ------------------------------------------------------------- block cache
// Released device blocks of at least kCacheMinBytes, per device and by size.
// A block enters the cache only when nothing can still use it (after a
// device or stream synchronisation), so it can be handed to any stream at
// once.  The maps are never destroyed (buffers may be released while the
// process exits).
constexpr size_t kCacheMinBytes = (size_t)4 << 20;
static std::mutex* g_cache_mu = new std::mutex;
static auto* g_cache = new std::map<int, std::multimap<size_t, void*>>;

// Sizes handed out by the cache: whole MiB, powers of two from 32 MiB up (so
// results that grow from call to call fit blocks released earlier).
static size_t cache_round(size_t n) {
  if (n >= kPoolRoundBytes) {
    size_t w = kPoolRoundBytes;
    while (w < n) w <<= 1;
    return w;
  }
  const size_t mib = (size_t)1 << 20;
  return (n + mib - 1) / mib * mib;
}

// Blocks released in stream order: they join the cache once their event
// (recorded on the releasing stream after its last use) has completed.
struct PendingBlock {
  void* p;
  size_t bytes;
  cudaEvent_t ev;
};
static auto* g_pending = new std::map<int, std::vector<PendingBlock>>;

static int pointer_device(void* p) {
  cudaPointerAttributes attr{};
  if (cudaPointerGetAttributes(&attr, p) == cudaSuccess) return attr.device;
  (void)cudaGetLastError();
  int dev = 0;
  cudaGetDevice(&dev);
  return dev;
}

static void cache_put(void* p, size_t bytes) {
  const int dev = pointer_device(p);
  std::lock_guard<std::mutex> lock(*g_cache_mu);
  (*g_cache)[dev].emplace(bytes, p);
}

// Releases a block once the work queued on `s` so far has completed (falls
// back to synchronising `s` when no event can be recorded).
static void cache_put_after(void* p, size_t bytes, cudaStream_t s) {
  cudaEvent_t ev = nullptr;
  if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess || cudaEventRecord(ev, s) != cudaSuccess) {
    (void)cudaGetLastError();
    if (ev) cudaEventDestroy(ev);
    cudaStreamSynchronize(s);
    cache_put(p, bytes);
    return;
  }
  const int dev = pointer_device(p);
  std::lock_guard<std::mutex> lock(*g_cache_mu);
  (*g_pending)[dev].push_back({p, bytes, ev});
}

// Moves the pending blocks of `dev` whose events completed (all of them when
// `all`, after the caller synchronised the device) into the cache; the
// caller holds the lock.
static void collect_pending(int dev, bool all) {
  auto& pend = (*g_pending)[dev];
  auto& m = (*g_cache)[dev];
  size_t keep = 0;
  for (size_t i = 0; i < pend.size(); ++i) {
    const cudaError_t q = all ? cudaSuccess : cudaEventQuery(pend[i].ev);
    if (q == cudaSuccess) {
      cudaEventDestroy(pend[i].ev);
      m.emplace(pend[i].bytes, pend[i].p);
    } else {
      if (q != cudaErrorNotReady) (void)cudaGetLastError();
      pend[keep++] = pend[i];
    }
  }
  pend.resize(keep);
}

// A cached block of the current device of at least n bytes and at most 2 n.
static void* cache_take(size_t n, size_t* got) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
  std::lock_guard<std::mutex> lock(*g_cache_mu);
  collect_pending(dev, false);
  auto& m = (*g_cache)[dev];
  auto it = m.lower_bound(n);
  if (it == m.end() || it->first > 2 * n) return nullptr;
  void* p = it->second;
  *got = it->first;
  m.erase(it);
  return p;
}

// Frees the current device's cached blocks.
static void cache_drain() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return;
  std::multimap<size_t, void*> blocks;
  {
    // the caller synchronised the device: every pending block is free
    std::lock_guard<std::mutex> lock(*g_cache_mu);
    collect_pending(dev, true);
    blocks.swap((*g_cache)[dev]);
  }
  for (auto& kv : blocks) cudaFree(kv.second);
}

void DevBuf::release() {
  if (!p) return;
  if (cached) {
    // nothing may use the block once it is back in the cache
    if (local) {
      cache_put_after(p, bytes, st);
    } else {
      cudaDeviceSynchronize();
      cache_put(p, bytes);
    }
  } else if (local) {
    cudaFreeAsync(p, st);
  } else {
    // same guarantee as cudaFree: nothing in flight still uses the memory
    cudaDeviceSynchronize();
    cudaFreeAsync(p, nullptr);
  }
  p = nullptr;
  bytes = 0;
  cached = false;
}

void DevBuf::release_synced() {
  if (!p) return;
  if (cached) {
    if (local) cache_put_after(p, bytes, st);
    else cache_put(p, bytes);
  } else {
    cudaFreeAsync(p, local ? st : nullptr);
  }
  p = nullptr;
  bytes = 0;
  cached = false;
}

int DevBuf::ensure(size_t n, cudaStream_t s) {
  if (n <= bytes && p) return 0;
  release();
  if (local) st = s;
  if (n == 0) n = 16;
  if (n >= kCacheMinBytes) {
    size_t want = cache_round(n), got = 0;
    void* q = cache_take(want, &got);
    if (!q) {
      cudaError_t e = cudaMalloc(&q, want);
      if (e == cudaErrorMemoryAllocation) {
        // give back what the cache and the pool hold and try again, at the
        // exact size last
        (void)cudaGetLastError();
        cudaDeviceSynchronize();
        cache_drain();
        cudaMemPool_t pool = nullptr;
        if (device_pool(&pool) == 0) cudaMemPoolTrimTo(pool, 0);
        e = cudaMalloc(&q, want);
        if (e == cudaErrorMemoryAllocation && want != n) {
          (void)cudaGetLastError();
          want = n;
          e = cudaMalloc(&q, want);
        }
      }
      if (e != cudaSuccess) {
        (void)cudaGetLastError();
        return fail(VBG_E_NOMEM, "device allocation of " + std::to_string(n) + " bytes failed (" +
                                     std::string(cudaGetErrorString(e)) + ")");
      }
      got = want;
    }
    p = q;
    bytes = got;
    cached = true;
    return 0;
  }
  cudaMemPool_t pool = nullptr;
  int rc = device_pool(&pool);
  if (rc) return rc;
  cudaError_t e = cudaMallocFromPoolAsync(&p, n, pool, s);
  if (e == cudaErrorMemoryAllocation) {
    // give back what the cache and the pool hold and try once more
    (void)cudaGetLastError();
    cudaDeviceSynchronize();
    cache_drain();
    cudaMemPoolTrimTo(pool, 0);
    e = cudaMallocFromPoolAsync(&p, n, pool, s);
  }
  if (e != cudaSuccess) {
    p = nullptr;
    (void)cudaGetLastError();
    return fail(VBG_E_NOMEM, "device allocation of " + std::to_string(n) + " bytes failed (" +
                                 std::string(cudaGetErrorString(e)) + ")");
  }
  bytes = n;
  cached = false;
  // an owned buffer may be used on any stream: wait for the allocation
  if (!local && s == nullptr) VBG_CUDA(cudaStreamSynchronize(nullptr));
  return 0;
}

int reserve_pool(size_t bytes) {
  cudaMemPool_t pool = nullptr;
  int rc = device_pool(&pool);
  if (rc) return rc;
  if (bytes == 0) return 0;
  // the pool keeps released memory up to its release threshold
  uint64_t thr = 0;
  VBG_CUDA(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr));
  if (bytes > thr) VBG_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &bytes));
  void* p = nullptr;
  VBG_CUDA(cudaMallocFromPoolAsync(&p, bytes, pool, nullptr));
  VBG_CUDA(cudaFreeAsync(p, nullptr));
  VBG_CUDA(cudaDeviceSynchronize());
  return 0;
}

int trim_pool() {
  cudaMemPool_t pool = nullptr;
  int rc = device_pool(&pool);
  if (rc) return rc;
  VBG_CUDA(cudaDeviceSynchronize());
  cache_drain();
  VBG_CUDA(cudaMemPoolTrimTo(pool, 0));
  return 0;
}

// Pinned host staging for device -> host structure copies (grows, never freed).
static std::mutex g_stage_mu;
static void* g_stage = nullptr;
static size_t g_stage_bytes = 0;

static int stage_ensure(size_t bytes) {
  if (bytes <= g_stage_bytes) return 0;
  if (g_stage) cudaFreeHost(g_stage);
  g_stage = nullptr;
  g_stage_bytes = 0;
  const size_t want = std::max(bytes + bytes / 2, (size_t)1 << 24);  // grow geometrically
  VBG_CUDA(cudaHostAlloc(&g_stage, want, cudaHostAllocDefault));
  g_stage_bytes = want;
  return 0;
}

template <typename T>
static int exclusive_sum(const T* in, T* out, int64_t n, cudaStream_t s) {
  size_t tmp = 0;
  VBG_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp, in, out, n, s));
  DevBuf t(s);
  int rc = t.ensure(std::max<size_t>(tmp, 16));
  if (rc) return rc;
  VBG_CUDA(cub::DeviceScan::ExclusiveSum(t.p, tmp, in, out, n, s));
  return 0;
}

int exclusive_sum_int(const int* in, int* out, int64_t n, cudaStream_t s) { return exclusive_sum(in, out, n, s); }

// Warp per block row: slot sizes (into size[slot]), gather metadata and the
// diagonal slot.  size has nnzb + 1 entries (the last one is set to 0).
__global__ void slot_info_kernel(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                                 const int* __restrict__ bsz, const int64_t* __restrict__ soff, int64_t nnzb,
                                 int64_t* __restrict__ size, int2* __restrict__ meta, int* __restrict__ diag) {
  const int lane = threadIdx.x & 31;
  const int warps = gridDim.x * (blockDim.x >> 5);
  for (int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); i < n; i += warps) {
    const int r = bsz[i];
    int d = -1;
    for (int e = rp[i] + lane; e < rp[i + 1]; e += 32) {
      const int j = ci[e];
      const int c = bsz[j];
      size[e] = (int64_t)r * c;
      meta[e] = make_int2(static_cast<int>(static_cast<uint32_t>(soff[j])),
                          static_cast<int>(((static_cast<uint32_t>(r) & 0xffu) << 8) | (static_cast<uint32_t>(c) & 0xffu)));
      if (j == i) d = e;
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) d = max(d, __shfl_xor_sync(0xffffffffu, d, off));
    if (lane == 0) diag[i] = d;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) size[nnzb] = 0;
}

int adopt_device_structure(vbg_matrix* m, const vbg_matrix* like, DevBuf& d_rp, DevBuf& d_ci, int64_t nnzb,
                           cudaStream_t s) {
  const int n = like->n;
  m->n = n;
  m->nnzb = nnzb;
  m->N = like->N;
  m->min_bs = like->min_bs;
  m->max_bs = like->max_bs;
  m->kind = like->kind;
  m->h_bsz = like->h_bsz;
  m->h_scal_off = like->h_scal_off;
  m->class_segs = like->class_segs;
  swap_mem(m->row_ptr, d_rp);
  swap_mem(m->col_ind, d_ci);
  int rc;
  if ((rc = m->bsz.ensure(std::max(n, 1) * sizeof(int), s))) return rc;
  if ((rc = m->scal_off.ensure((n + 1) * sizeof(int64_t), s))) return rc;
  if ((rc = m->row_perm.ensure(std::max(n, 1) * sizeof(int), s))) return rc;
  if ((rc = m->diag_slot.ensure(std::max(n, 1) * sizeof(int), s))) return rc;
  if (n) {
    VBG_CUDA(cudaMemcpyAsync(m->bsz.p, like->bsz.p, n * sizeof(int), cudaMemcpyDeviceToDevice, s));
    VBG_CUDA(cudaMemcpyAsync(m->row_perm.p, like->row_perm.p, n * sizeof(int), cudaMemcpyDeviceToDevice, s));
  }
  VBG_CUDA(cudaMemcpyAsync(m->scal_off.p, like->scal_off.p, (n + 1) * sizeof(int64_t), cudaMemcpyDeviceToDevice, s));
  DevBuf sizes(s);
  if ((rc = sizes.ensure((nnzb + 1) * sizeof(int64_t)))) return rc;
  if ((rc = m->blk_off.ensure((nnzb + 1) * sizeof(int64_t), s))) return rc;
  if ((rc = m->slot_meta.ensure(std::max<int64_t>(nnzb, 1) * sizeof(int2), s))) return rc;
  const int grid = std::max(1, std::min((n + 7) / 8, sm_count() * 16));
  slot_info_kernel<<<grid, 256, 0, s>>>(n, m->row_ptr.as<int>(), m->col_ind.as<int>(), m->bsz.as<int>(),
                                        m->scal_off.as<int64_t>(), nnzb, sizes.as<int64_t>(),
                                        m->slot_meta.as<int2>(), m->diag_slot.as<int>());
  VBG_CUDA(cudaGetLastError());
  if ((rc = exclusive_sum(sizes.as<int64_t>(), m->blk_off.as<int64_t>(), nnzb + 1, s))) return rc;
  // the host mirrors are read back on first use
  m->h_row_ptr.clear();
  m->h_col_ind.clear();
  m->h_blk_off.clear();
  m->h_row_ptr.shrink_to_fit();
  m->h_col_ind.shrink_to_fit();
  m->h_blk_off.shrink_to_fit();
  m->host_struct = false;
  m->dup_cols = like->dup_cols;
  VBG_CUDA(cudaMemcpyAsync(&m->nnz, m->blk_off.as<int64_t>() + nnzb, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
  VBG_CUDA(cudaStreamSynchronize(s));
  m->invalidate_structure();
  return 0;
}

// Slot sizes, per-slot gather records, diagonal slots and value offsets of m
// from its device row pointers, columns, block sizes and scalar offsets
// (validated by the caller); m->nnz is read back.
int device_slot_structure(vbg_matrix* m, cudaStream_t s) {
  const int n = m->n;
  const int64_t nnzb = m->nnzb;
  int rc;
  DevBuf sizes(s);
  if ((rc = sizes.ensure((nnzb + 1) * sizeof(int64_t)))) return rc;
  if ((rc = m->blk_off.ensure((nnzb + 1) * sizeof(int64_t), s))) return rc;
  if ((rc = m->slot_meta.ensure(std::max<int64_t>(nnzb, 1) * sizeof(int2), s))) return rc;
  if ((rc = m->diag_slot.ensure(std::max(n, 1) * sizeof(int), s))) return rc;
  const int grid = std::max(1, std::min((n + 7) / 8, sm_count() * 16));
  slot_info_kernel<<<grid, 256, 0, s>>>(n, m->row_ptr.as<int>(), m->col_ind.as<int>(), m->bsz.as<int>(),
                                        m->scal_off.as<int64_t>(), nnzb, sizes.as<int64_t>(),
                                        m->slot_meta.as<int2>(), m->diag_slot.as<int>());
  VBG_CUDA(cudaGetLastError());
  if ((rc = exclusive_sum(sizes.as<int64_t>(), m->blk_off.as<int64_t>(), nnzb + 1, s))) return rc;
  VBG_CUDA(cudaMemcpyAsync(&m->nnz, m->blk_off.as<int64_t>() + nnzb, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
  VBG_CUDA(cudaStreamSynchronize(s));
  return 0;
}

int ensure_host_structure(const vbg_matrix* cm, cudaStream_t s) {
  auto* m = const_cast<vbg_matrix*>(cm);
  if (m->host_struct) return 0;
  const int n = m->n;
  const int64_t nnzb = m->nnzb;
  std::lock_guard<std::mutex> lock(g_stage_mu);
  const size_t b_rp = (n + 1) * sizeof(int), b_ci = nnzb * sizeof(int), b_off = (nnzb + 1) * sizeof(int64_t);
  int rc;
  if ((rc = stage_ensure(b_off + b_rp + b_ci + 64))) return rc;
  char* st = static_cast<char*>(g_stage);
  VBG_CUDA(cudaMemcpyAsync(st, m->blk_off.p, b_off, cudaMemcpyDeviceToHost, s));
  VBG_CUDA(cudaMemcpyAsync(st + b_off, m->row_ptr.p, b_rp, cudaMemcpyDeviceToHost, s));
  if (nnzb) VBG_CUDA(cudaMemcpyAsync(st + b_off + b_rp, m->col_ind.p, b_ci, cudaMemcpyDeviceToHost, s));
  VBG_CUDA(cudaStreamSynchronize(s));
  const int64_t* off = reinterpret_cast<const int64_t*>(st);
  m->h_blk_off.assign(off, off + nnzb + 1);
  const int* rpp = reinterpret_cast<const int*>(st + b_off);
  m->h_row_ptr.assign(rpp, rpp + n + 1);
  const int* cip = reinterpret_cast<const int*>(st + b_off + b_rp);
  m->h_col_ind.assign(cip, cip + nnzb);
  m->host_struct = true;
  return 0;
}

// ------------------------------------------------------------- column view
__global__ void col_count_kernel(const int* __restrict__ ci, int64_t nnzb, int* __restrict__ cnt) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nnzb; e += (int64_t)gridDim.x * blockDim.x)
    atomicAdd(&cnt[ci[e]], 1);
}

__global__ void iota_kernel(int* __restrict__ v, int64_t n) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x)
    v[e] = (int)e;
}

// Warp per block row: row_of[slot] = row.
__global__ void row_of_slot_kernel(int n, const int* __restrict__ rp, int* __restrict__ row_of) {
  const int lane = threadIdx.x & 31;
  const int warps = gridDim.x * (blockDim.x >> 5);
  for (int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); i < n; i += warps)
    for (int p = rp[i] + lane; p < rp[i + 1]; p += 32) row_of[p] = i;
}

__global__ void gather_int_kernel(const int* __restrict__ src, const int* __restrict__ idx, int64_t n,
                                  int* __restrict__ dst) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x)
    dst[e] = src[idx[e]];
}

// Column view for the adjoint apply and SpGEMM: for each block column j the
// slots (i, j) by increasing slot -- increasing row -- (csc_slot) with their
// rows (csc_row), csc_ptr the column starts; csc_perm the identity order of
// the columns.  The slots are sorted by column with a stable radix sort, so
// each column keeps the row order of the row-major layout (the reference's
// column-incoming plan, vbcsr/core/detail/backend/vbcsr_backend.hpp:543-625).
int build_csc_dev(const vbg_matrix* cm, cudaStream_t s) {
  auto* m = const_cast<vbg_matrix*>(cm);
  if (m->csc_valid) return 0;
  const int n = m->n;
  const int64_t nnzb = m->nnzb;
  int rc;
  if ((rc = m->csc_ptr.ensure((n + 1) * sizeof(int), s))) return rc;
  if ((rc = m->csc_slot.ensure(std::max<int64_t>(nnzb, 1) * sizeof(int), s))) return rc;
  if ((rc = m->csc_row.ensure(std::max<int64_t>(nnzb, 1) * sizeof(int), s))) return rc;
  if ((rc = m->csc_perm.ensure(std::max(n, 1) * sizeof(int), s))) return rc;
  DevBuf cnt(s), keys_out(s), iota(s), row_of(s), tmp(s);
  if ((rc = cnt.ensure((n + 1) * sizeof(int)))) return rc;
  VBG_CUDA(cudaMemsetAsync(cnt.p, 0, (n + 1) * sizeof(int), s));
  const int g = (int)std::max<int64_t>(1, std::min<int64_t>((nnzb + 255) / 256, sm_count() * 16));
  if (nnzb) {
    col_count_kernel<<<g, 256, 0, s>>>(m->col_ind.as<int>(), nnzb, cnt.as<int>());
    VBG_CUDA(cudaGetLastError());
  }
  if ((rc = exclusive_sum(cnt.as<int>(), m->csc_ptr.as<int>(), n + 1, s))) return rc;
  if (n) {
    iota_kernel<<<std::max(1, std::min((n + 255) / 256, sm_count() * 8)), 256, 0, s>>>(m->csc_perm.as<int>(), n);
    VBG_CUDA(cudaGetLastError());
  }
  if (nnzb) {
    if ((rc = keys_out.ensure(nnzb * sizeof(int)))) return rc;
    if ((rc = iota.ensure(nnzb * sizeof(int)))) return rc;
    if ((rc = row_of.ensure(nnzb * sizeof(int)))) return rc;
    iota_kernel<<<g, 256, 0, s>>>(iota.as<int>(), nnzb);
    row_of_slot_kernel<<<std::max(1, std::min((n + 7) / 8, sm_count() * 16)), 256, 0, s>>>(n, m->row_ptr.as<int>(),
                                                                                        row_of.as<int>());
    VBG_CUDA(cudaGetLastError());
    int bits = 1;
    while (bits < 31 && (1 << bits) < n) ++bits;
    size_t tb = 0;
    VBG_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb, m->col_ind.as<int>(), keys_out.as<int>(), iota.as<int>(),
                                             m->csc_slot.as<int>(), nnzb, 0, bits, s));
    if ((rc = tmp.ensure(std::max<size_t>(tb, 16)))) return rc;
    VBG_CUDA(cub::DeviceRadixSort::SortPairs(tmp.p, tb, m->col_ind.as<int>(), keys_out.as<int>(), iota.as<int>(),
                                             m->csc_slot.as<int>(), nnzb, 0, bits, s));
    gather_int_kernel<<<g, 256, 0, s>>>(row_of.as<int>(), m->csc_slot.as<int>(), nnzb, m->csc_row.as<int>());
    VBG_CUDA(cudaGetLastError());
  }
  m->csc_valid = true;
  return 0;
}

__global__ void flags_kernel(const unsigned char* __restrict__ keep, int64_t n, int* __restrict__ flags) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i <= n; i += (int64_t)gridDim.x * blockDim.x)
    flags[i] = i < n ? (keep[i] ? 1 : 0) : 0;
}

__global__ void compact_pattern_kernel(int n, const int* __restrict__ rp, const int* __restrict__ ci, int64_t nnzb,
                                       const unsigned char* __restrict__ keep, const int* __restrict__ pos,
                                       int* __restrict__ new_rp, int* __restrict__ new_ci, int* __restrict__ old_of) {
  const int64_t tid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t e = tid; e < nnzb; e += stride)
    if (keep[e]) {
      new_ci[pos[e]] = ci[e];
      old_of[pos[e]] = (int)e;
    }
  for (int64_t i = tid; i <= n; i += stride) new_rp[i] = pos[rp[i]];
}

template <typename T>
__global__ void gather_blocks_kernel(int64_t nout, const int* __restrict__ old_of, const int64_t* __restrict__ old_off,
                                     const T* __restrict__ src, const int64_t* __restrict__ new_off,
                                     T* __restrict__ dst) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t k = blockIdx.x * (int64_t)(blockDim.x >> 5) + (threadIdx.x >> 5); k < nout; k += warps) {
    const int64_t o = old_off[old_of[k]], d = new_off[k], len = new_off[k + 1] - d;
    for (int64_t e = lane; e < len; e += 32) dst[d + e] = src[o + e];
  }
}

// Keeps the slots with keep[slot] != 0 (device flags), structure built on the device.
int compact_by_mask_dev(vbg_matrix* m, const unsigned char* keep, cudaStream_t s) {
  const int64_t nnzb = m->nnzb;
  if (nnzb == 0) return 0;
  int rc;
  DevBuf flags(s), pos(s);
  if ((rc = flags.ensure((nnzb + 1) * sizeof(int)))) return rc;
  if ((rc = pos.ensure((nnzb + 1) * sizeof(int)))) return rc;
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((nnzb + 256) / 256, sm_count() * 16));
  flags_kernel<<<grid, 256, 0, s>>>(keep, nnzb, flags.as<int>());
  VBG_CUDA(cudaGetLastError());
  if ((rc = exclusive_sum(flags.as<int>(), pos.as<int>(), nnzb + 1, s))) return rc;
  int kept = 0;
  VBG_CUDA(cudaMemcpyAsync(&kept, pos.as<int>() + nnzb, sizeof(int), cudaMemcpyDeviceToHost, s));
  VBG_CUDA(cudaStreamSynchronize(s));
  if (kept == nnzb) return 0;
  DevBuf new_rp(s), new_ci(s), old_of(s);
  if ((rc = new_rp.ensure((m->n + 1) * sizeof(int)))) return rc;
  if ((rc = new_ci.ensure(std::max(kept, 1) * sizeof(int)))) return rc;
  if ((rc = old_of.ensure(std::max(kept, 1) * sizeof(int)))) return rc;
  compact_pattern_kernel<<<grid, 256, 0, s>>>(m->n, m->row_ptr.as<int>(), m->col_ind.as<int>(), nnzb, keep,
                                              pos.as<int>(), new_rp.as<int>(), new_ci.as<int>(), old_of.as<int>());
  VBG_CUDA(cudaGetLastError());
  auto d = std::make_unique<vbg_matrix>();
  d->dtype = m->dtype;
  d->device = m->device;
  if ((rc = adopt_device_structure(d.get(), m, new_rp, new_ci, kept, s))) return rc;
  const size_t es = elem_size(d->dtype);
  if ((rc = d->vals.ensure(std::max<int64_t>(d->nnz, 1) * es, s))) return rc;
  if (kept) {
    const int g2 = (int)std::max<int64_t>(1, std::min<int64_t>((kept + 7) / 8, sm_count() * 16));
    if (d->dtype == VBG_C128)
      gather_blocks_kernel<cplx><<<g2, 256, 0, s>>>(kept, old_of.as<int>(), m->blk_off.as<int64_t>(),
                                                    m->vals.as<cplx>(), d->blk_off.as<int64_t>(), d->vals.as<cplx>());
    else
      gather_blocks_kernel<double><<<g2, 256, 0, s>>>(kept, old_of.as<int>(), m->blk_off.as<int64_t>(),
                                                      m->vals.as<double>(), d->blk_off.as<int64_t>(),
                                                      d->vals.as<double>());
    VBG_CUDA(cudaGetLastError());
  }
  // old_of and the old values are released when this returns / m's buffers move
  VBG_CUDA(cudaStreamSynchronize(s));
  move_into(m, d.get());
  return 0;
}

}  // namespace vbg

extern "C" int vbg_memory_reserve(size_t bytes) { return vbg::reserve_pool(bytes); }
extern "C" int vbg_memory_trim(void) { return vbg::trim_pool(); }
