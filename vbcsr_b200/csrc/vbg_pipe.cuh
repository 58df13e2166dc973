// Pipelined forward multivector apply.  Included by vbg_apply.cu inside
// namespace vbg, after ApplyArgs, the scalar helpers and grid_reduce2.
//
// Y = A X (+ the fused epilogue of vbg_cheb_step) for multivectors whose
// padded row is a whole number of warp widths (ld a multiple of 32 * PipeEV)
// and whose blocks are at most 8 x 8.
//
// One warp streams the spans of a tile of kPipeRows consecutive block rows.
// A span is a run of stored blocks of one block row with consecutive block
// columns (at most `cap` X rows): its X rows and its kernel-layout values
// (column by column, 16-byte padded) are each contiguous, so it is multiplied
// as one r x c block.  For every span, one lane has the bulk-copy engine move
// the c rows of X and the values into a stage of a per-warp ring in shared memory,
// up to kPipeStages - 1 blocks ahead of the block the warp multiplies; the stage's
// mbarrier counts the bytes in.  The copies cost the warp a few instructions
// per block instead of one per lane and row, and the gathers of several
// blocks are in flight while the FMAs of the current one issue.  Tiles go
// round-robin over the warps of the grid, so all warps sweep the matrix
// together and the rows of X shared between neighbouring tiles stay in L2;
// rows are visited in natural order (one launch for all block sizes), so X is
// streamed from HBM once per apply.
//
// Every wait on a stage is bounded (kPipeWaitNs).  A wait that runs out sets
// bit 0 of g_pipe_status (read by vbg_device_status), the warp stops issuing
// and multiplying, waits (bounded again) for the copies it still has in
// flight and leaves; the launch then completes with wrong values and the
// status bit set instead of hanging.

constexpr int kPipeWarps = 4;
#ifndef VBG_PIPE_STAGES
#define VBG_PIPE_STAGES 4
#endif
#ifndef VBG_PIPE_BATCH
#define VBG_PIPE_BATCH 2
#endif
constexpr int kPipeStages = VBG_PIPE_STAGES;  // a power of two
constexpr int kPipeBatch = VBG_PIPE_BATCH;    // blocks armed per producer pass (<= kPipeStages / 2)
constexpr int kPipeRows = 4;
#ifndef VBG_PIPE_CAP
#define VBG_PIPE_CAP 5
#endif
constexpr int kPipeSpanCap = VBG_PIPE_CAP;  // X rows per span, raised to the largest block
constexpr int kPipeMaxBs = 8;
constexpr unsigned long long kPipeWaitNs = 1000000000ull;

// Scalars per lane and X row piece: 16 bytes for FP64 and complex, 8 for FP32
// (so that a 64-column FP32 multivector still spans one warp).
template <typename T> struct PipeEV { static constexpr int v = sizeof(T) >= 16 ? 1 : 2; };

template <typename T, int EV>
struct alignas(EV * sizeof(T)) PipeLane {
  T v[EV];
};

template <typename T>
struct alignas(16) Vec16 {
  static constexpr int N = sizeof(T) >= 16 ? 1 : 16 / (int)sizeof(T);
  T v[N];
};

// Bit 0: a pipelined apply gave up waiting for a stage.
__device__ unsigned g_pipe_status;

__device__ __forceinline__ unsigned smem_addr(const void* p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(unsigned bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(count) : "memory");
}
// Makes barrier initialisation visible to the bulk-copy (async) proxy.
__device__ __forceinline__ void mbar_init_fence() {
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}
// Orders this thread's earlier shared-memory accesses before later bulk
// copies into the same memory.
__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}
// One arrival that also expects `bytes` to be delivered by bulk copies.
__device__ __forceinline__ void mbar_arm(unsigned bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.release.cta.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(bytes)
               : "memory");
}
// Global -> shared bulk copy completing on `bar` (no multicast).  Both
// addresses 16-byte aligned, `bytes` a multiple of 16.
__device__ __forceinline__ void bulk_g2s(unsigned dst, const void* src, unsigned bytes, unsigned bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}
// Asks L2 to fetch [src, src + bytes) (16-byte aligned, multiple of 16).
__device__ __forceinline__ void bulk_prefetch_l2(const void* src, unsigned bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;\n" ::"l"(src), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;\n" : "=l"(t));
  return t;
}
// Waits (all lanes) for the phase of `bar` with the given parity, at most
// kPipeWaitNs; warp-uniform result.
__device__ __forceinline__ bool pipe_wait(unsigned bar, unsigned parity) {
  bool ok = mbar_try_wait(bar, parity);
  if (!ok) {
    const unsigned long long t0 = global_ns();
    while (!(ok = mbar_try_wait(bar, parity)))
      if (global_ns() - t0 > kPipeWaitNs) break;
  }
  return __all_sync(0xffffffffu, ok);
}

// Shared memory of one warp: X ring, value ring, stage barriers, block widths.
template <typename T>
__host__ __device__ constexpr size_t pipe_xstage_bytes(int cm) {
  return (size_t)cm * 32 * PipeEV<T>::v * sizeof(T);
}
template <typename T>
__host__ __device__ constexpr size_t pipe_warp_bytes(int cm) {
  return kPipeStages * pipe_xstage_bytes<T>(cm) + (size_t)kPipeStages * 64 * sizeof(T) + kPipeStages * 8 +
         ((kPipeStages * 4 + 15) / 16) * 16;
}

// One warp's view of its pipeline.
template <typename T, int EV>
struct PipeCtx {
  const unsigned char* xlane;  // this lane's piece of stage 0, row 0 of the X ring
  const T* vring;              // values of stage 0
  int* width;                  // per stage: columns of the staged block
  unsigned xring_s, vring_s, bar_s;  // shared-window addresses of the rings and barriers
  int xstage;                  // bytes of one X stage
  int lane, n, nitems, nchunks, nw;
};

// Arms the stages for the spans in consumption order (this warp's items,
// their rows in order, each row's spans in order), kPipeBatch spans at a
// time: lane j arms the stage of the j-th span of the batch and issues its
// copies, so one pass of warp instructions stages several spans.  The span
// records of the next batch and the span range of the next item are loaded
// one step ahead, so arming a batch does not wait on global memory.
template <typename T, int EV>
struct PipeProducer {
  int item, e, end, v0;
  int stage;       // stage of the next span to arm
  int ahead;       // stages armed and not yet consumed
  int ne, nend;    // span range of item + nw (loaded ahead)
  int pe;          // first span of the prefetched batch records (-1: none)
  int4 psp;        // this lane's prefetched span record
  long long pvo;   // and its kernel-layout value offset

  __device__ __forceinline__ void load_bounds(const ApplyArgs& a, const PipeCtx<T, EV>& cx, int it) {
    ne = nend = 0;
    if (it < cx.nitems) {
      const int r0 = (it / cx.nchunks) * kPipeRows, r1 = min(r0 + kPipeRows, cx.n);
      ne = a.row_sptr[r0];
      nend = a.row_sptr[r1];
    }
  }
  __device__ __forceinline__ void load_records(const ApplyArgs& a, const PipeCtx<T, EV>& cx, int at, int stop) {
    pe = at;
    if (at + cx.lane < stop) {
      psp = a.spans[at + cx.lane];
      pvo = std::is_same<T, float>::value ? a.span_koff32[at + cx.lane]
                                          : (static_cast<long long>(psp.w) << 32) | static_cast<unsigned>(psp.z);
    }
  }

  __device__ __forceinline__ void next(const ApplyArgs& a, const T* __restrict__ vals, const PipeCtx<T, EV>& cx) {
    constexpr int LB = EV * sizeof(T);
    if (ahead > kPipeStages - 1 - kPipeBatch) return;  // no room for a batch
    while (e == end) {  // step to the next item with spans
      if (item + cx.nw >= cx.nitems) return;
      item += cx.nw;
      e = ne;
      end = nend;
      v0 = (item % cx.nchunks) * 32 * EV;
      load_bounds(a, cx, item + cx.nw);
    }
    const int cnt = min(kPipeBatch, end - e);
    if (pe != e) load_records(a, cx, e, end);
    if (cx.lane < cnt) {
      const int4 sp = psp;
      const long long vo = pvo;
      const int c = sp.y & 0xff;                                         // X rows of the span
      const int nv = c * kernel_layout_rows(sp.y >> 8, (int)sizeof(T));  // its kernel-layout scalars
      const int st = (stage + cx.lane) & (kPipeStages - 1);
      const unsigned bar = cx.bar_s + st * 8;
      const unsigned xdst = cx.xring_s + st * cx.xstage;
      const unsigned xbytes = c * 32 * LB, vbytes = nv * (unsigned)sizeof(T);
      cx.width[st] = c;
      fence_proxy_async();  // the warp's reads of this stage's previous span come first
      mbar_arm(bar, xbytes + vbytes);
      const T* X = static_cast<const T*>(a.X);
      if (cx.nchunks == 1) {
        bulk_g2s(xdst, X + (long long)sp.x * a.ld, xbytes, bar);  // c whole rows, contiguous
      } else {
        for (int q = 0; q < c; ++q)
          bulk_g2s(xdst + q * 32 * LB, X + (long long)(sp.x + q) * a.ld + v0, 32 * LB, bar);
      }
      bulk_g2s(cx.vring_s + st * 64 * (unsigned)sizeof(T), vals + vo, vbytes, bar);
    }
    e += cnt;
    stage = (stage + cnt) & (kPipeStages - 1);
    ahead += cnt;
    // the next batch's records: the rest of this item, else the next item's start
    if (e < end) load_records(a, cx, e, end);
    else load_records(a, cx, ne, nend);
  }
};

// acc[o] += sum_q A[o][q] X[q] over one staged R x C block: values in the
// kernel layout (column q = A[0..R)[q], padded to RP scalars) at vs, this
// lane's pieces of the C rows of X at xs.  Fully unrolled: every shared
// memory read has an immediate offset.
template <typename T, int EV, int R, int C>
__device__ __forceinline__ void pipe_block_rc(const unsigned char* xs, const T* vs,
                                              PipeLane<T, EV> (&acc)[kPipeMaxBs]) {
  using L = PipeLane<T, EV>;
  using V = Vec16<T>;
  constexpr int RP = kernel_layout_rows(R, (int)sizeof(T));
#pragma unroll
  for (int q = 0; q < C; ++q) {
    const L x = *reinterpret_cast<const L*>(xs + q * 32 * sizeof(L));
#pragma unroll
    for (int j = 0; j < RP / V::N; ++j) {
      const V w = reinterpret_cast<const V*>(vs + q * RP)[j];
#pragma unroll
      for (int t = 0; t < V::N; ++t) {
        if (j * V::N + t < R) {
#pragma unroll
          for (int u = 0; u < EV; ++u) acc[j * V::N + t].v[u] = fma_s(w.v[t], x.v[u], acc[j * V::N + t].v[u]);
        }
      }
    }
  }
}

template <typename T, int EV, int R>
__device__ __forceinline__ void pipe_block(int c, const unsigned char* xs, const T* vs,
                                           PipeLane<T, EV> (&acc)[kPipeMaxBs]) {
  switch (c) {  // 1 <= c <= kPipeMaxBs
    case 1: pipe_block_rc<T, EV, R, 1>(xs, vs, acc); break;
    case 2: pipe_block_rc<T, EV, R, 2>(xs, vs, acc); break;
    case 3: pipe_block_rc<T, EV, R, 3>(xs, vs, acc); break;
    case 4: pipe_block_rc<T, EV, R, 4>(xs, vs, acc); break;
    case 5: pipe_block_rc<T, EV, R, 5>(xs, vs, acc); break;
    case 6: pipe_block_rc<T, EV, R, 6>(xs, vs, acc); break;
    case 7: pipe_block_rc<T, EV, R, 7>(xs, vs, acc); break;
    default: pipe_block_rc<T, EV, R, 8>(xs, vs, acc); break;
  }
}

// One block row of r scalar rows: multiply its blocks [e, e1) from the ring
// (the producer keeps between kPipeStages - 1 - kPipeBatch and
// kPipeStages - 1 blocks staged ahead), then the epilogue.
// Only the block product is specialised on r: one copy of the block loop
// keeps the kernel's register count that of its largest block product.
// Returns false when a stage wait ran out (the warp then stops).
template <typename T, int EV>
__device__ __forceinline__ bool pipe_row(const ApplyArgs& a, const T* __restrict__ vals, PipeProducer<T, EV>& prod,
                                         const PipeCtx<T, EV>& cx, int r, int e, int e1, int& c_stage,
                                         unsigned& phase, long long y0, int v0, double& d0, double& d1) {
  using L = PipeLane<T, EV>;
  if (cx.lane == 0 && cx.nchunks == 1) {
    // the epilogue's streamed operands come from HBM: have L2 fetch this
    // row's slices while its spans are multiplied
    const unsigned bytes = (unsigned)(r * a.ld * sizeof(T));
    if (a.gamma != 0.0) bulk_prefetch_l2(static_cast<const T*>(a.Xprev) + y0 * a.ld, bytes);
    if (a.want_dots && a.dotw) bulk_prefetch_l2(static_cast<const T*>(a.dotw) + y0 * a.ld, bytes);
  }
  L acc[kPipeMaxBs];
#pragma unroll
  for (int o = 0; o < kPipeMaxBs; ++o)
#pragma unroll
    for (int u = 0; u < EV; ++u) acc[o].v[u] = zero_s<T>();
  for (; e < e1; ++e) {
    prod.next(a, vals, cx);
    if (!pipe_wait(cx.bar_s + c_stage * 8, (phase >> c_stage) & 1u)) return false;
    phase ^= 1u << c_stage;
    --prod.ahead;
    const int c = cx.width[c_stage];
    const unsigned char* xs = cx.xlane + c_stage * cx.xstage;
    const T* vs = cx.vring + c_stage * 64;
    switch (r) {  // 1 <= r <= kPipeMaxBs
      case 1: pipe_block<T, EV, 1>(c, xs, vs, acc); break;
      case 2: pipe_block<T, EV, 2>(c, xs, vs, acc); break;
      case 3: pipe_block<T, EV, 3>(c, xs, vs, acc); break;
      case 4: pipe_block<T, EV, 4>(c, xs, vs, acc); break;
      case 5: pipe_block<T, EV, 5>(c, xs, vs, acc); break;
      case 6: pipe_block<T, EV, 6>(c, xs, vs, acc); break;
      case 7: pipe_block<T, EV, 7>(c, xs, vs, acc); break;
      default: pipe_block<T, EV, 8>(c, xs, vs, acc); break;
    }
    __syncwarp();  // all lanes are done with this stage before it is refilled
    c_stage = (c_stage + 1) & (kPipeStages - 1);
  }
  const T* X = static_cast<const T*>(a.X);
#pragma unroll
  for (int o = 0; o < kPipeMaxBs; ++o) {
    if (o >= r) break;
    const long long el = (y0 + o) * a.ld + v0 + cx.lane * EV;
    L y;
    if (a.beta == 0.0 && a.gamma == 0.0 && !a.want_dots && !a.acc) {
#pragma unroll
      for (int u = 0; u < EV; ++u) y.v[u] = scal_r(a.alpha, acc[o].v[u]);
    } else {
      L xs, xp, xd, ac;
      if (a.beta != 0.0 || (a.want_dots && !a.dotw)) xs = *reinterpret_cast<const L*>(X + el);
      if (a.gamma != 0.0) xp = *reinterpret_cast<const L*>(static_cast<const T*>(a.Xprev) + el);
      if (a.want_dots) xd = a.dotw ? *reinterpret_cast<const L*>(static_cast<const T*>(a.dotw) + el) : xs;
      if (a.acc) ac = *reinterpret_cast<const L*>(static_cast<const T*>(a.acc) + el);
#pragma unroll
      for (int u = 0; u < EV; ++u) {
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
      if (a.acc) *reinterpret_cast<L*>(static_cast<T*>(a.acc) + el) = ac;
    }
    *reinterpret_cast<L*>(static_cast<T*>(a.Y) + el) = y;
    // one output row at a time: keeps the loads of later rows from being
    // hoisted (and held in registers) across this row's stores
    asm volatile("" ::: "memory");
  }
  return true;
}

template <typename T, int EV>
__global__ void __launch_bounds__(kPipeWarps * 32) apply_pipe_kernel(ApplyArgs a, const T* __restrict__ vals, int cm,
                                                                     int nchunks, int part_base, int total) {
  extern __shared__ __align__(16) unsigned char pipe_smem[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  PipeCtx<T, EV> cx;
  unsigned char* wbase = pipe_smem + (size_t)warp * pipe_warp_bytes<T>(cm);
  cx.xstage = (int)pipe_xstage_bytes<T>(cm);
  cx.xlane = wbase + lane * EV * sizeof(T);
  T* vring = reinterpret_cast<T*>(wbase + kPipeStages * cx.xstage);
  cx.vring = vring;
  unsigned char* bars = reinterpret_cast<unsigned char*>(vring + kPipeStages * 64);
  cx.width = reinterpret_cast<int*>(bars + kPipeStages * 8);
  cx.xring_s = smem_addr(wbase);
  cx.vring_s = smem_addr(vring);
  cx.bar_s = smem_addr(bars);
  cx.lane = lane;
  cx.n = a.n_rows;
  cx.nchunks = nchunks;
  cx.nitems = ((cx.n + kPipeRows - 1) / kPipeRows) * nchunks;
  cx.nw = gridDim.x * kPipeWarps;
  const int gw = blockIdx.x * kPipeWarps + warp;
  const int* __restrict__ bsz = a.bsz;
  const int64_t* __restrict__ soff = a.scal_off;

  if (lane == 0) {
    for (int s = 0; s < kPipeStages; ++s) mbar_init(cx.bar_s + s * 8, 1);
    mbar_init_fence();
  }
  __syncwarp();

  PipeProducer<T, EV> prod;
  prod.item = gw - cx.nw;
  prod.e = prod.end = prod.v0 = prod.stage = prod.ahead = 0;
  prod.pe = -1;
  prod.load_bounds(a, cx, gw);
  prod.next(a, vals, cx);

  int c_stage = 0;
  unsigned phase = 0;
  bool alive = true;
  double d0 = 0.0, d1 = 0.0;
  // row records of an item's tile, one row per lane (loaded one item ahead)
  auto load_tile = [&](int it, int& e0, int& e1, int& r, long long& y) {
    if (it >= cx.nitems) return;
    const int q0 = (it / nchunks) * kPipeRows, q1 = min(q0 + kPipeRows, cx.n);
    if (lane < q1 - q0) {
      e0 = a.row_sptr[q0 + lane];
      e1 = a.row_sptr[q0 + lane + 1];
      r = bsz[q0 + lane];
      y = soff[q0 + lane];
    }
  };
  int n_e0 = 0, n_e1 = 0, n_r = 0;
  long long n_y = 0;
  load_tile(gw, n_e0, n_e1, n_r, n_y);
  for (int item = gw; alive && item < cx.nitems; item += cx.nw) {
    const int tile = item / nchunks;
    const int v0 = (item - tile * nchunks) * 32 * EV;
    const int n = cx.n;
    const int r0 = tile * kPipeRows, r1 = min(r0 + kPipeRows, n);
    const int t_e0 = n_e0, t_e1 = n_e1, t_r = n_r;
    const long long t_y = n_y;
    load_tile(item + cx.nw, n_e0, n_e1, n_r, n_y);
    int e = __shfl_sync(0xffffffffu, t_e0, 0);
    for (int li = 0; li < r1 - r0; ++li) {
      const int e1 = __shfl_sync(0xffffffffu, t_e1, li);
      const int r = __shfl_sync(0xffffffffu, t_r, li);
      const long long y0 = __shfl_sync(0xffffffffu, t_y, li);
      double rd0 = 0.0, rd1 = 0.0;
      if (!pipe_row<T, EV>(a, vals, prod, cx, r, e, e1, c_stage, phase, y0, v0, a.row_dots ? rd0 : d0,
                           a.row_dots ? rd1 : d1)) {
        alive = false;
        break;
      }
      if (a.want_dots && a.row_dots) write_row_dots(a.row_dots, r0 + li, rd0, rd1);
      e = e1;
    }
  }
  if (!alive) {
    if (lane == 0) atomicOr(&g_pipe_status, 1u);
    // let the copies still in flight land before the shared memory is released
    for (int k = 0; k < prod.ahead; ++k) {
      const int s = (c_stage + k) & (kPipeStages - 1);
      pipe_wait(cx.bar_s + s * 8, (phase >> s) & 1u);
    }
  }
  if (a.want_dots && !a.row_dots) grid_reduce2(d0, d1, a.partials, a.counter, a.dots_out, part_base, total);
}
