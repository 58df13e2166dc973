// Pipelined forward multivector apply.  Included by vbg_apply.cu inside
// namespace vbg, after ApplyArgs, the scalar helpers and grid_reduce2.
//
// Y = A X (+ the fused epilogue of vbg_cheb_step) for multivectors whose
// padded row is a whole number of lane-group widths and whose blocks are at
// most 8 x 8.
//
// One warp streams the spans of a tile of kPipeRows consecutive block rows.
// A span is a run of stored blocks of one block row with consecutive block
// columns (at most `cap` X rows): its X rows and its kernel-layout values
// (column by column, 16-byte padded) are each contiguous, so it is multiplied
// as one r x c block.  For every span, one lane has the bulk-copy engine move
// the c rows of X and the values into a stage of a per-warp ring in shared
// memory, a batch of spans ahead of the ones the warp multiplies; the stage's
// mbarrier counts the bytes in.  The copies cost the warp a few instructions
// per span instead of one per lane and row, and the gathers of several spans
// are in flight while the FMAs of the current ones issue.
//
// Lane groups: the 32 lanes form G groups of L = 32 / G lanes; a group's lanes
// cover W = L * EV columns of the multivector (16-byte pieces for FP64 and
// complex, 8-byte for FP32).  G = 1 when a row of X is at least a warp wide
// (k = 64 FP64); for narrower multivectors (k = 16, 32) the G groups multiply
// G different spans of the same block row at once and their partial sums
// are added by a butterfly at the end of the row.
//
// Tiles go round-robin over the warps of the grid, so all warps sweep the
// matrix together and the rows of X shared between neighbouring tiles stay in
// L2; rows are visited in natural order (one launch for all block sizes), so
// X is streamed from HBM once per apply.
//
// Every wait on a stage is bounded (kPipeWaitNs).  A wait that runs out sets
// bit 0 of g_pipe_status (read by vbg_device_status), the warp stops issuing
// and multiplying, waits (bounded again) for the copies it still has in
// flight and leaves; the launch then completes with wrong values and the
// status bit set instead of hanging.

constexpr int kPipeWarps = 4;
constexpr int kPipeRows = 4;
#ifndef VBG_PIPE_CAP
#define VBG_PIPE_CAP 5
#endif
constexpr int kPipeSpanCap = VBG_PIPE_CAP;  // X rows per span, raised to the largest block
constexpr int kPipeMaxBs = 8;
constexpr unsigned long long kPipeWaitNs = 1000000000ull;

// Ring shape per lane-group count: stages (a power of two) and spans armed
// per producer pass; a round of the consumer takes G stages.
template <int G>
struct PipeShape {
  static constexpr int S = G >= 4 ? 8 : 4;
  static constexpr int B = G >= 4 ? 4 : 2;
  static constexpr int L = 32 / G;
};

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
// Global -> shared bulk copy completing on `bar`, to this CTA only.  Both
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
// This lane waits for the phase of `bar` with the given parity, at most
// kPipeWaitNs.
__device__ __forceinline__ bool mbar_wait_bounded(unsigned bar, unsigned parity) {
  bool ok = mbar_try_wait(bar, parity);
  if (!ok) {
    const unsigned long long t0 = global_ns();
    while (!(ok = mbar_try_wait(bar, parity)))
      if (global_ns() - t0 > kPipeWaitNs) break;
  }
  return ok;
}
// Whole warp, warp-uniform result.
__device__ __forceinline__ bool pipe_wait(unsigned bar, unsigned parity) {
  return __all_sync(0xffffffffu, mbar_wait_bounded(bar, parity));
}

// Shared memory of one warp: X ring, value ring, stage barriers, span widths.
template <typename T, int G>
__host__ __device__ constexpr size_t pipe_xstage_bytes(int cm) {
  return (size_t)cm * PipeShape<G>::L * PipeEV<T>::v * sizeof(T);
}
template <typename T, int G>
__host__ __device__ constexpr size_t pipe_warp_bytes(int cm) {
  return PipeShape<G>::S * pipe_xstage_bytes<T, G>(cm) + (size_t)PipeShape<G>::S * 64 * sizeof(T) +
         PipeShape<G>::S * 8 + ((PipeShape<G>::S * 4 + 15) / 16) * 16;
}

// One warp's view of its pipeline.
template <typename T, int EV>
struct PipeCtx {
  const unsigned char* xlane;  // this lane's piece (within its group) of stage 0, row 0 of the X ring
  const T* vring;              // values of stage 0
  int* width;                  // per stage: X rows of the staged span
  unsigned xring_s, vring_s, bar_s;  // shared-window addresses of the rings and barriers
  int xstage;                  // bytes of one X stage
  int lane, n, nitems, nchunks, nw;
};

// Arms the stages for the spans in consumption order (this warp's items,
// their rows in order, each row's spans in order), B spans at a time: lane j
// arms the stage of the j-th span of the batch and issues its copies, so one
// pass of warp instructions stages several spans.  The span records of the
// next batch and the span range of the next item are loaded one step ahead,
// so arming a batch does not wait on global memory.
template <typename T, int EV, int G>
struct PipeProducer {
  static constexpr int S = PipeShape<G>::S, B = PipeShape<G>::B, L = PipeShape<G>::L;
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
    if (cx.lane < B && at + cx.lane < stop) {
      psp = a.spans[at + cx.lane];
      pvo = std::is_same<T, float>::value ? a.span_koff32[at + cx.lane]
                                          : (static_cast<long long>(psp.w) << 32) | static_cast<unsigned>(psp.z);
    }
  }

  __device__ __forceinline__ void next(const ApplyArgs& a, const T* __restrict__ vals, const PipeCtx<T, EV>& cx) {
    constexpr int LB = EV * sizeof(T);
    // room for a batch: whole-warp rows keep one stage free, the lane-group
    // shapes may fill the ring (a round consumes G stages)
    if (ahead > S - (G == 1 ? 1 : 0) - B) return;
    while (e == end) {          // step to the next item with spans
      if (item + cx.nw >= cx.nitems) return;
      item += cx.nw;
      e = ne;
      end = nend;
      v0 = (item % cx.nchunks) * L * EV;
      load_bounds(a, cx, item + cx.nw);
    }
    const int cnt = min(B, end - e);
    if (pe != e) load_records(a, cx, e, end);
    if (cx.lane < cnt) {
      const int4 sp = psp;
      const long long vo = pvo;
      const int c = sp.y & 0xff;                                         // X rows of the span
      const int nv = c * kernel_layout_rows(sp.y >> 8, (int)sizeof(T));  // its kernel-layout scalars
      const int st = (stage + cx.lane) & (S - 1);
      const unsigned bar = cx.bar_s + st * 8;
      const unsigned xdst = cx.xring_s + st * cx.xstage;
      const unsigned xbytes = c * L * LB, vbytes = nv * (unsigned)sizeof(T);
      cx.width[st] = c;
      fence_proxy_async();  // the warp's reads of this stage's previous span come first
      mbar_arm(bar, xbytes + vbytes);
      const T* X = static_cast<const T*>(a.X);
      if (cx.nchunks == 1) {
        bulk_g2s(xdst, X + (long long)sp.x * a.ld, xbytes, bar);  // c whole rows, contiguous
      } else {
        for (int q = 0; q < c; ++q)
          bulk_g2s(xdst + q * L * LB, X + (long long)(sp.x + q) * a.ld + v0, L * LB, bar);
      }
      bulk_g2s(cx.vring_s + st * 64 * (unsigned)sizeof(T), vals + vo, vbytes, bar);
    }
    e += cnt;
    stage = (stage + cnt) & (S - 1);
    ahead += cnt;
    // the next batch's records: the rest of this item, else the next item's start
    if (e < end) load_records(a, cx, e, end);
    else load_records(a, cx, ne, nend);
  }
};

// acc[o] += sum_q A[o][q] X[q] over one staged R x C span: values in the
// kernel layout (column q = A[0..R)[q], padded to RP scalars) at vs, this
// lane's pieces of the C rows of X at xs (row stride LBR bytes).  Fully
// unrolled: every shared memory read has an immediate offset.  With lane
// groups the warp runs the widest span of its groups (C = cmax) and a lane
// skips the columns q >= c of its own span (PRED).
template <typename T, int EV, int R, int C, bool PRED>
__device__ __forceinline__ void pipe_block_rc(const unsigned char* xs, const T* vs, int c, int LBR,
                                              PipeLane<T, EV> (&acc)[kPipeMaxBs]) {
  using L = PipeLane<T, EV>;
  using V = Vec16<T>;
  constexpr int RP = kernel_layout_rows(R, (int)sizeof(T));
#pragma unroll
  for (int q = 0; q < C; ++q) {
    if (PRED && q >= c) continue;
    const L x = *reinterpret_cast<const L*>(xs + q * LBR);
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

template <typename T, int EV, int R, bool PRED>
__device__ __forceinline__ void pipe_block(int cmax, int c, const unsigned char* xs, const T* vs, int LBR,
                                           PipeLane<T, EV> (&acc)[kPipeMaxBs]) {
  switch (cmax) {  // 1 <= cmax <= kPipeMaxBs
    case 1: pipe_block_rc<T, EV, R, 1, PRED>(xs, vs, c, LBR, acc); break;
    case 2: pipe_block_rc<T, EV, R, 2, PRED>(xs, vs, c, LBR, acc); break;
    case 3: pipe_block_rc<T, EV, R, 3, PRED>(xs, vs, c, LBR, acc); break;
    case 4: pipe_block_rc<T, EV, R, 4, PRED>(xs, vs, c, LBR, acc); break;
    case 5: pipe_block_rc<T, EV, R, 5, PRED>(xs, vs, c, LBR, acc); break;
    case 6: pipe_block_rc<T, EV, R, 6, PRED>(xs, vs, c, LBR, acc); break;
    case 7: pipe_block_rc<T, EV, R, 7, PRED>(xs, vs, c, LBR, acc); break;
    default: pipe_block_rc<T, EV, R, 8, PRED>(xs, vs, c, LBR, acc); break;
  }
}

// One block row of r scalar rows: multiply its spans [e, e1) from the ring,
// G at a time (one per lane group), the producer keeping a batch staged
// ahead; add the groups' partial sums; epilogue by group 0.  Only the span
// product is specialised on r: one copy of the loop keeps the kernel's
// register count that of its largest product.  Returns false when a stage
// wait ran out (the warp then stops).
template <typename T, int EV, int G>
__device__ __forceinline__ bool pipe_row(const ApplyArgs& a, const T* __restrict__ vals, PipeProducer<T, EV, G>& prod,
                                         const PipeCtx<T, EV>& cx, int r, int e, int e1, int& c_stage,
                                         unsigned& phase, long long y0, int v0, double& d0, double& d1) {
  using L = PipeLane<T, EV>;
  constexpr int S = PipeShape<G>::S, LN = PipeShape<G>::L;
  constexpr int LBR = LN * (int)sizeof(L);  // bytes of one staged X row
  constexpr bool PRED = G > 1;
  const int grp = cx.lane / LN;
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
  if constexpr (G == 1) {
    // one span at a time (a row of X is a whole warp wide)
    for (; e < e1; ++e) {
      prod.next(a, vals, cx);
      if (!pipe_wait(cx.bar_s + c_stage * 8, (phase >> c_stage) & 1u)) return false;
      phase ^= 1u << c_stage;
      --prod.ahead;
      const int c = cx.width[c_stage];
      const unsigned char* xs = cx.xlane + c_stage * cx.xstage;
      const T* vs = cx.vring + c_stage * 64;
      switch (r) {  // 1 <= r <= kPipeMaxBs
        case 1: pipe_block<T, EV, 1, false>(c, c, xs, vs, LBR, acc); break;
        case 2: pipe_block<T, EV, 2, false>(c, c, xs, vs, LBR, acc); break;
        case 3: pipe_block<T, EV, 3, false>(c, c, xs, vs, LBR, acc); break;
        case 4: pipe_block<T, EV, 4, false>(c, c, xs, vs, LBR, acc); break;
        case 5: pipe_block<T, EV, 5, false>(c, c, xs, vs, LBR, acc); break;
        case 6: pipe_block<T, EV, 6, false>(c, c, xs, vs, LBR, acc); break;
        case 7: pipe_block<T, EV, 7, false>(c, c, xs, vs, LBR, acc); break;
        default: pipe_block<T, EV, 8, false>(c, c, xs, vs, LBR, acc); break;
      }
      __syncwarp();  // all lanes are done with this stage before it is refilled
      c_stage = (c_stage + 1) & (S - 1);
    }
  } else {
  for (; e < e1; e += G) {
    prod.next(a, vals, cx);
    const int nact = min(G, e1 - e);
    const bool active = grp < nact;
    const int st = (c_stage + grp) & (S - 1);
    const bool ok = active ? mbar_wait_bounded(cx.bar_s + st * 8, (phase >> st) & 1u) : true;
    if (!__all_sync(0xffffffffu, ok)) return false;
#pragma unroll
    for (int g = 0; g < G; ++g)
      if (g < nact) phase ^= 1u << ((c_stage + g) & (S - 1));
    prod.ahead -= nact;
    const int c = active ? cx.width[st] : 0;
    int cmax = c;
    if (G > 1) cmax = __reduce_max_sync(0xffffffffu, c);
    const unsigned char* xs = cx.xlane + st * cx.xstage;
    const T* vs = cx.vring + st * 64;
    switch (r) {  // 1 <= r <= kPipeMaxBs
      case 1: pipe_block<T, EV, 1, PRED>(cmax, c, xs, vs, LBR, acc); break;
      case 2: pipe_block<T, EV, 2, PRED>(cmax, c, xs, vs, LBR, acc); break;
      case 3: pipe_block<T, EV, 3, PRED>(cmax, c, xs, vs, LBR, acc); break;
      case 4: pipe_block<T, EV, 4, PRED>(cmax, c, xs, vs, LBR, acc); break;
      case 5: pipe_block<T, EV, 5, PRED>(cmax, c, xs, vs, LBR, acc); break;
      case 6: pipe_block<T, EV, 6, PRED>(cmax, c, xs, vs, LBR, acc); break;
      case 7: pipe_block<T, EV, 7, PRED>(cmax, c, xs, vs, LBR, acc); break;
      default: pipe_block<T, EV, 8, PRED>(cmax, c, xs, vs, LBR, acc); break;
    }
    __syncwarp();  // all lanes are done with these stages before they are refilled
    c_stage = (c_stage + nact) & (S - 1);
  }
  }
  if (G > 1) {
#pragma unroll
    for (int o = 0; o < kPipeMaxBs; ++o) {
      if (o >= r) break;
#pragma unroll
      for (int off = LN; off < 32; off <<= 1)
#pragma unroll
        for (int u = 0; u < EV; ++u) acc[o].v[u] = add_s(acc[o].v[u], shfl_xor_s(acc[o].v[u], off));
    }
    if (grp != 0) return true;
  }
  const T* X = static_cast<const T*>(a.X);
#pragma unroll
  for (int o = 0; o < kPipeMaxBs; ++o) {
    if (o >= r) break;
    const long long el = (y0 + o) * a.ld + v0 + (cx.lane % LN) * EV;
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

template <typename T, int EV, int G>
__global__ void __launch_bounds__(kPipeWarps * 32) apply_pipe_kernel(ApplyArgs a, const T* __restrict__ vals, int cm,
                                                                     int nchunks, int part_base, int total) {
  constexpr int S = PipeShape<G>::S, LN = PipeShape<G>::L;
  extern __shared__ __align__(16) unsigned char pipe_smem[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  PipeCtx<T, EV> cx;
  unsigned char* wbase = pipe_smem + (size_t)warp * pipe_warp_bytes<T, G>(cm);
  cx.xstage = (int)pipe_xstage_bytes<T, G>(cm);
  cx.xlane = wbase + (lane % LN) * EV * sizeof(T);
  T* vring = reinterpret_cast<T*>(wbase + S * cx.xstage);
  cx.vring = vring;
  unsigned char* bars = reinterpret_cast<unsigned char*>(vring + S * 64);
  cx.width = reinterpret_cast<int*>(bars + S * 8);
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
    for (int s = 0; s < S; ++s) mbar_init(cx.bar_s + s * 8, 1);
    mbar_init_fence();
  }
  __syncwarp();

  PipeProducer<T, EV, G> prod;
  prod.item = gw - cx.nw;
  prod.e = prod.end = prod.v0 = prod.stage = prod.ahead = 0;
  prod.pe = -1;
  prod.load_bounds(a, cx, gw);
  for (int k = 0; k < (G == 1 ? 1 : S / PipeShape<G>::B); ++k) prod.next(a, vals, cx);

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
  int c_stage = 0;
  unsigned phase = 0;
  bool alive = true;
  double d0 = 0.0, d1 = 0.0;
  for (int item = gw; alive && item < cx.nitems; item += cx.nw) {
    const int tile = item / nchunks;
    const int v0 = (item - tile * nchunks) * LN * EV;
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
      if (!pipe_row<T, EV, G>(a, vals, prod, cx, r, e, e1, c_stage, phase, y0, v0, rd0, rd1)) {
        alive = false;
        break;
      }
      if (a.want_dots) {
        if (a.row_dots) {
          write_row_dots(a.row_dots, r0 + li, rd0, rd1);
        } else {
          d0 += rd0;
          d1 += rd1;
        }
      }
      e = e1;
    }
  }
  if (!alive) {
    if (lane == 0) atomicOr(&g_pipe_status, 1u);
    // let the copies still in flight land before the shared memory is released
    for (int k = 0; k < prod.ahead; ++k) {
      const int s = (c_stage + k) & (S - 1);
      pipe_wait(cx.bar_s + s * 8, (phase >> s) & 1u);
    }
  }
  if (a.want_dots && !a.row_dots) grid_reduce2(d0, d1, a.partials, a.counter, a.dots_out, part_base, total);
}
