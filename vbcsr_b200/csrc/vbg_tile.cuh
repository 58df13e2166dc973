// Row-tiled forward multivector apply.  Included by vbg_apply.cu inside
// namespace vbg, after vbg_pipe.cuh (it uses the pipe's block product,
// mbarrier helpers and bulk copies).
//
// Y = A X (+ the fused epilogue of vbg_cheb_step) for multivectors whose
// padded row is exactly one warp of 16-byte (FP64, complex) or 8-byte (FP32)
// pieces -- k = 64 FP64 / FP32, k = 32 complex -- and blocks of at most
// 8 x 8, when the matrix's rows can be cut into tiles whose working set fits
// shared memory.
//
// A tile is up to kTileRowsMax consecutive block rows.  The block columns its
// blocks touch form a few contiguous ranges for matrices whose neighbours
// sit at nearby indices (lattice and banded orderings: about three ranges,
// the tile's own strip and its neighbour strips); the union of their X rows
// is staged once per tile, instead of each block row gathering its
// neighbours' rows (2.5-3.5 times fewer bytes between L2 and the SMs), and so
// are the tile's values in the kernel layout and its q-list.  One thread
// arms the tile's mbarrier, issues a bulk copy per range, one for the values
// and one for the q-list, and asks L2 to fetch the tile's Xprev and
// dot-partner rows, which the epilogue reads from global memory.
//
// The q-list of a block row holds, for every X row its blocks read in
// column order, that row's place in the staged X (16-bit, read four at a
// time).  A warp walks it with one shared-memory load of the lane's piece of
// X, the column's values (a broadcast) and R x EV multiply-adds per X row:
// no per-block records, shuffles or switches.  For multivectors of half a
// warp's width (16 FP64 or FP32 columns) two lane groups each take every
// other X row and add their sums by a shuffle.
//
// The host plans the tiles once per structure (tile_plan): the tallest
// height in {16, 12, 10, 8, 6, 4} whose largest tile fits the budget, each
// tile's ranges with their place in shared memory, the q-lists, a record per
// block row, and the tile's rows cut into kTileWarps runs of consecutive rows
// of about equal work (balanced_runs), one per warp.  Matrices whose tiles do
// not fit (neighbours far apart) keep the pipelined apply.
//
// Every wait is bounded (kPipeWaitNs); a timeout sets bit 0 of
// g_pipe_status, and the CTA waits (bounded) for its copies and leaves.
// Only warp 0 polls the tile's mbarrier; the others wait at the CTA barrier
// (polling by all warps cost more issue slots than the tile's arithmetic).

constexpr int kTileWarps = 8;                      // warps of a tile CTA
constexpr int kTileRowsMax = 16;                   // block rows per tile, in up to kTileWarps runs
constexpr size_t kTileSmemBudget = 113 * 1024;     // shared memory per CTA: two CTAs per SM (228 KB)
constexpr size_t kTileSmemBudget32 = 75 * 1024;    // FP32 values: three CTAs per SM
constexpr int kTileMaxRanges = 64;                 // bulk copies of X per tile

// Shared memory of a tile CTA: barrier, values (vcap scalars of `ves`
// bytes), the q-list (qcap bytes), X rows (xcap rows of rb bytes).
__host__ __device__ inline size_t tile_vals_bytes(int64_t vcap, int ves) {
  return ((size_t)vcap * ves + 15) / 16 * 16;
}
__host__ __device__ inline size_t tile_smem_bytes(int64_t vcap, int ves, int qcap, int xcap, int rb) {
  return 16 + tile_vals_bytes(vcap, ves) + (size_t)qcap + (size_t)xcap * rb;
}

// Splits the block rows [0, T) of a tile (work w[i] each) into at most W
// runs of consecutive rows with the smallest largest run; bounds[k] is the
// end of run k (runs k >= the number used are empty).  T <= kTileRowsMax.
static void balanced_runs(const int64_t* w, int T, int W, int* bounds) {
  int64_t pre[kTileRowsMax + 1] = {0};
  for (int i = 0; i < T; ++i) pre[i + 1] = pre[i] + w[i];
  // best[k][j]: smallest largest run splitting rows [0, j) into k runs
  int64_t best[kTileWarps + 1][kTileRowsMax + 1];
  int cut[kTileWarps + 1][kTileRowsMax + 1];
  for (int j = 0; j <= T; ++j) {
    best[1][j] = pre[j];
    cut[1][j] = 0;
  }
  const int K = std::min(W, std::max(T, 1));
  for (int k = 2; k <= K; ++k)
    for (int j = 0; j <= T; ++j) {
      best[k][j] = best[k - 1][j];
      cut[k][j] = j;
      for (int i = 0; i < j; ++i) {
        const int64_t v = std::max(best[k - 1][i], pre[j] - pre[i]);
        if (v < best[k][j]) {
          best[k][j] = v;
          cut[k][j] = i;
        }
      }
    }
  int end = T;
  for (int k = K; k >= 1; --k) {
    bounds[k - 1] = end;
    end = k > 1 ? cut[k][end] : 0;
  }
  for (int k = K; k < W; ++k) bounds[k] = T;
}

// The q-list layout (plan independent): block row i's entries start at
// qstart[i], a multiple of 4 (so a row's entries load four at a time as one
// 8-byte vector), and number qn[i] = the X rows its blocks read.
static void qlist_layout(const vbg_matrix* m, std::vector<int>& qstart, std::vector<int>& qn) {
  const int n = m->n;
  qstart.assign(n + 1, 0);
  qn.assign(n, 0);
  for (int i = 0; i < n; ++i) {
    int c = 0;
    for (int p = m->h_row_ptr[i]; p < m->h_row_ptr[i + 1]; ++p) c += m->h_bsz[m->h_col_ind[p]];
    qn[i] = c;
    qstart[i + 1] = qstart[i] + ((c + 3) & ~3);
  }
}
// The staged q-list slice of the tile of block rows [t0, t1): entries
// [qbase, qend) rounded out to 16-byte boundaries (8 entries).
static inline int qlist_base(const std::vector<int>& qstart, int t0) { return qstart[t0] & ~7; }
static inline int qlist_bytes(const std::vector<int>& qstart, int t0, int t1) {
  return 2 * (((qstart[t1] + 7) & ~7) - (qstart[t0] & ~7));
}

// Plans the row tiles of matrix m for X rows of rb bytes and values of ves
// bytes (kernel layout), tiles of at most `cap` block rows.  *out is the
// plan, or nullptr when no tile height fits the budget.  Needs the spans (ensure_spans); reads the host
// structure.
static int tile_plan(const vbg_matrix* cm, int rb, int ves, cudaStream_t s, TilePlan** out,
                     int cap = kTileRowsMax) {
  auto* m = const_cast<vbg_matrix*>(cm);
  *out = nullptr;
  const auto key = std::make_tuple(rb, ves, cap);
  auto found = m->tile_plans.find(key);
  if (found != m->tile_plans.end()) {
    if (found->second->rows > 0) *out = found->second.get();
    return 0;
  }
  VBG_CHECK(m->span_cap > 0 && (int64_t)m->h_span_x.size() == m->nspans, VBG_E_STATE, "tile plan needs the spans");
  int rc = ensure_host_structure(m, s);
  if (rc) return rc;
  const int n = m->n;
  const std::vector<int>& rp = m->h_row_ptr;
  const std::vector<int>& ci = m->h_col_ind;
  const std::vector<int>& bsz = m->h_bsz;
  const std::vector<int64_t>& soff = m->h_scal_off;
  // value scalars of each block row in the kernel layout
  std::vector<int64_t> vrow(n, 0);
  for (int i = 0; i < n; ++i) {
    const int rpad = kernel_layout_rows(bsz[i], ves);
    for (int p = rp[i]; p < rp[i + 1]; ++p) vrow[i] += (int64_t)bsz[ci[p]] * rpad;
  }
  std::vector<int> stamp(n, -1), cols;
  std::vector<int4> ranges;  // of one tile: {first column, last column, ., .}
  // The tile [t0, t1): its distinct block columns merged into runs of
  // consecutive columns; returns the staged X rows.
  auto tile_ranges = [&](int tid, int t0, int t1) -> int64_t {
    cols.clear();
    for (int i = t0; i < t1; ++i)  // the tile's own rows of X (the epilogue's beta X)
      if (stamp[i] != tid) {
        stamp[i] = tid;
        cols.push_back(i);
      }
    for (int p = rp[t0]; p < rp[t1]; ++p)
      if (stamp[ci[p]] != tid) {
        stamp[ci[p]] = tid;
        cols.push_back(ci[p]);
      }
    std::sort(cols.begin(), cols.end());
    ranges.clear();
    for (int c : cols) {
      if (!ranges.empty() && c == ranges.back().y + 1) ranges.back().y = c;
      else ranges.push_back(make_int4(c, c, 0, 0));
    }
    int64_t xr = 0;
    for (const int4& g : ranges) xr += soff[g.y + 1] - soff[g.x];
    return xr;
  };
  std::vector<int> qstart, qn;
  qlist_layout(m, qstart, qn);
  auto plan = std::make_unique<TilePlan>();
  int tag = 0;
  // the tallest tile (at most `cap` block rows) whose largest staging fits
  // the budget
  for (int tr : {16, 12, 10, 8, 6, 4}) {
    if (tr > cap) continue;
    bool fits = true;
    int64_t xcap = 0, vcap = 0, ocap = 0;
    int qcap = 0;
    for (int t0 = 0; t0 < n && fits; t0 += tr) {
      const int t1 = std::min(n, t0 + tr);
      const int64_t xr = tile_ranges(tag++, t0, t1);
      int64_t vs = 0;
      for (int i = t0; i < t1; ++i) vs += vrow[i];
      xcap = std::max(xcap, xr);
      vcap = std::max(vcap, vs);
      ocap = std::max(ocap, soff[t1] - soff[t0]);
      qcap = std::max(qcap, qlist_bytes(qstart, t0, t1));
      // shared-memory rows are 16-bit q-list entries
      fits = (int)ranges.size() <= kTileMaxRanges && xcap <= 65535 &&
             tile_smem_bytes(vcap, ves, qcap, (int)xcap, rb) <= (ves == 4 ? kTileSmemBudget32 : kTileSmemBudget);
    }
    if (fits) {
      plan->rows = tr;
      plan->xcap = (int)xcap;
      plan->vcap = vcap;
      plan->owncap = (int)ocap;
      plan->qcap = qcap;
      break;
    }
  }
  if (plan->rows == 0) {  // remembered as infeasible
    m->tile_plans[key] = std::move(plan);
    return 0;
  }
  const int tr = plan->rows;
  const int ntiles = (n + tr - 1) / tr;
  std::vector<int4> h_tiles(4 * (size_t)ntiles), h_ranges, h_rowinfo(std::max(n, 1));
  // the q-list, padded so that the last tile's staged slice stays inside
  std::vector<unsigned short> h_qidx(((size_t)qstart[n] + 7) / 8 * 8 + 8, 0);
  int64_t k0 = 0;  // kernel-layout value offset of the tile's first slot
  for (int t = 0; t < ntiles; ++t) {
    const int t0 = t * tr, t1 = std::min(n, t0 + tr);
    tile_ranges(tag++, t0, t1);
    const int rbeg = (int)h_ranges.size();
    int dst = 0;
    for (const int4& g : ranges) {
      const int src = (int)soff[g.x], cnt = (int)(soff[g.y + 1] - soff[g.x]);
      h_ranges.push_back(make_int4(src, cnt, dst, 0));
      dst += cnt;
    }
    const int rend = (int)h_ranges.size();
    // the shared-memory row of a staged X row
    auto srow_of = [&](int x) {
      int lo = rbeg, hi = rend - 1;
      while (lo < hi) {
        const int mid = (lo + hi + 1) / 2;
        if (h_ranges[mid].x <= x) lo = mid;
        else hi = mid - 1;
      }
      return h_ranges[lo].z + (x - h_ranges[lo].x);
    };
    // every block row's q-list: the shared-memory row of each X row its
    // blocks read (a block column's rows lie in one range)
    const int qb = qlist_base(qstart, t0);
    int64_t vs = 0;
    for (int i = t0; i < t1; ++i) {
      int k = qstart[i];
      for (int p = rp[i]; p < rp[i + 1]; ++p) {
        const int x0 = (int)soff[ci[p]];
        for (int q = 0; q < bsz[ci[p]]; ++q) h_qidx[k++] = (unsigned short)srow_of(x0 + q);
      }
      h_rowinfo[i] = make_int4(qstart[i] - qb, qn[i], (int)vs, bsz[i]);
      vs += vrow[i];
    }
    // the tile's rows in runs of consecutive rows, one run per warp, with
    // balanced work (the multiply-adds and loads of a row: its X rows times
    // its size plus a few)
    int64_t wk[kTileRowsMax];
    for (int i = t0; i < t1; ++i) wk[i - t0] = (int64_t)qn[i] * (bsz[i] + 2) + 8;
    int bounds[kTileWarps];
    balanced_runs(wk, t1 - t0, kTileWarps, bounds);
    unsigned packed[2] = {0u, 0u};
    for (int w = 0; w < kTileWarps; ++w) packed[w / 4] |= (unsigned)bounds[w] << (8 * (w % 4));
    const int ys0 = (int)soff[t0], own = (int)(soff[t1] - soff[t0]);
    h_tiles[4 * (size_t)t] = make_int4(t0, t1, rbeg, rend);
    h_tiles[4 * (size_t)t + 1] = make_int4((int)(k0 & 0xffffffff), (int)(k0 >> 32), (int)(vs * ves), dst * rb);
    h_tiles[4 * (size_t)t + 2] = make_int4(srow_of(ys0), own, ys0, 0);
    h_tiles[4 * (size_t)t + 3] = make_int4(qb, qlist_bytes(qstart, t0, t1), (int)packed[0], (int)packed[1]);
    k0 += vs;
  }
  plan->ntiles = ntiles;
  plan->smem = (int)tile_smem_bytes(plan->vcap, ves, plan->qcap, plan->xcap, rb);
  if ((rc = plan->tiles.ensure(h_tiles.size() * sizeof(int4), s))) return rc;
  if ((rc = plan->ranges.ensure(std::max<size_t>(h_ranges.size(), 1) * sizeof(int4), s))) return rc;
  if ((rc = plan->qidx.ensure(h_qidx.size() * sizeof(unsigned short), s))) return rc;
  if ((rc = plan->rowinfo.ensure(h_rowinfo.size() * sizeof(int4), s))) return rc;
  VBG_CUDA(cudaMemcpyAsync(plan->tiles.p, h_tiles.data(), h_tiles.size() * sizeof(int4), cudaMemcpyHostToDevice, s));
  if (!h_ranges.empty())
    VBG_CUDA(cudaMemcpyAsync(plan->ranges.p, h_ranges.data(), h_ranges.size() * sizeof(int4), cudaMemcpyHostToDevice,
                             s));
  VBG_CUDA(cudaMemcpyAsync(plan->qidx.p, h_qidx.data(), h_qidx.size() * sizeof(unsigned short),
                           cudaMemcpyHostToDevice, s));
  VBG_CUDA(cudaMemcpyAsync(plan->rowinfo.p, h_rowinfo.data(), h_rowinfo.size() * sizeof(int4), cudaMemcpyHostToDevice,
                           s));
  if ((rc = plan->queue.ensure(2 * sizeof(int), s))) return rc;
  VBG_CUDA(cudaMemsetAsync(plan->queue.p, 0, 2 * sizeof(int), s));
  VBG_CUDA(cudaStreamSynchronize(s));  // the host vectors are locals
  *out = plan.get();
  m->tile_plans[key] = std::move(plan);
  return 0;
}

// Epilogue of one block row of the tiled applies (the pipelined apply's, for
// a warp-wide row): Y = alpha acc + beta X + gamma Xprev, the dots,
// acc += c Y.  The row's own X rows come from shared memory (xo: this lane's
// piece of the row's first scalar row, rows RB bytes apart); Xprev, the dot
// partner, the accumulator and Y are global (read once per apply; L2 has
// been asked to fetch the tile's rows).
// With G lane groups (a row of X is 32 / G lanes wide) every group holds the
// whole sum; group g writes the output rows o = g (mod G), `lane` is the
// lane within the group.
template <typename T, int EV, int RB, int G = 1>
__device__ __forceinline__ void tile_epilogue(const ApplyArgs& a, const PipeLane<T, EV> (&acc)[kPipeMaxBs], int r,
                                              long long y0, int lane, const unsigned char* xo, double& d0,
                                              double& d1, int grp = 0) {
  using L = PipeLane<T, EV>;
#pragma unroll
  for (int o = 0; o < kPipeMaxBs; ++o) {
    if (o >= r) break;
    if (G > 1 && o % G != grp) continue;
    const long long el = (y0 + o) * a.ld + lane * EV;
    L y;
    if (a.beta == 0.0 && a.gamma == 0.0 && !a.want_dots && !a.acc) {
#pragma unroll
      for (int u = 0; u < EV; ++u) y.v[u] = scal_r(a.alpha, acc[o].v[u]);
    } else {
      L xs, xp, xd, ac;
      if (a.beta != 0.0 || (a.want_dots && !a.dotw)) xs = *reinterpret_cast<const L*>(xo + o * RB);
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
  }
}

// One block row of R scalar rows out of shared memory into acc (zeroed
// here), by its q-list: ql holds the shared-memory rows of the nq X rows its
// blocks read (in slot order, column order within a block), four per 8-byte
// load; vr its values in the kernel layout (column q at vr + q * RP).  Per X
// row: one load of this lane's piece of the row, the column's R values
// (broadcast) and R x EV multiply-adds -- no per-block bookkeeping.  With G
// lane groups (narrow multivectors: a row of X is 32 / G lanes wide) group
// g takes the X rows q = g (mod G) and the groups' sums are added at the
// end, so every group holds the row's result.
template <typename T, int EV, int R, int G = 1>
__device__ __forceinline__ void qlist_row(const unsigned short* ql, int nq, const T* vr, const unsigned char* xl,
                                          PipeLane<T, EV> (&acc)[kPipeMaxBs], int grp = 0) {
  using L = PipeLane<T, EV>;
  using V = Vec16<T>;
  constexpr int RB = 32 / G * (int)sizeof(L);
  constexpr int RP = kernel_layout_rows(R, (int)sizeof(T));
  // FP32 at one scalar per lane: every four X rows summed on their own,
  // then added to the row's sum (two-level summation keeps the rounding
  // error of long rows near that of the pipelined apply's lane-group sums)
  constexpr bool kTwoLevel = std::is_same<T, float>::value && EV == 1;
#pragma unroll
  for (int o = 0; o < kPipeMaxBs; ++o)
#pragma unroll
    for (int u = 0; u < EV; ++u) acc[o].v[u] = zero_s<T>();
  L part[kTwoLevel ? R : 1];
  auto step = [&](int idx, const T* w, L (&dst)[kTwoLevel ? R : kPipeMaxBs]) {
    const L x = *reinterpret_cast<const L*>(xl + idx * RB);
#pragma unroll
    for (int j = 0; j < RP / V::N; ++j) {
      const V wv = reinterpret_cast<const V*>(w)[j];
#pragma unroll
      for (int t = 0; t < V::N; ++t) {
        if (j * V::N + t < R) {
#pragma unroll
          for (int u = 0; u < EV; ++u) dst[j * V::N + t].v[u] = fma_s(wv.v[t], x.v[u], dst[j * V::N + t].v[u]);
        }
      }
    }
  };
  // four q-list entries: this group's ones are q = grp, grp + G, ... < cnt
  auto group = [&](const ushort4 id, const T* w, int cnt) {
    auto entry = [&](int k) -> int { return k == 0 ? id.x : k == 1 ? id.y : k == 2 ? id.z : id.w; };
    if constexpr (kTwoLevel) {
#pragma unroll
      for (int o = 0; o < R; ++o)
#pragma unroll
        for (int u = 0; u < EV; ++u) part[o].v[u] = zero_s<T>();
    }
#pragma unroll
    for (int j = 0; j < 4; j += G) {
      const int k = j + (G > 1 ? grp : 0);
      if (k < cnt) {
        if constexpr (kTwoLevel) step(entry(k), w + k * RP, part);
        else step(entry(k), w + k * RP, acc);
      }
    }
    if constexpr (kTwoLevel) {
#pragma unroll
      for (int o = 0; o < R; ++o)
#pragma unroll
        for (int u = 0; u < EV; ++u) acc[o].v[u] += part[o].v[u];
    }
  };
  int q = 0;
  for (; q + 4 <= nq; q += 4) group(*reinterpret_cast<const ushort4*>(ql + q), vr + q * RP, 4);
  if (q < nq) group(*reinterpret_cast<const ushort4*>(ql + q), vr + q * RP, nq - q);
  if constexpr (G > 1) {
#pragma unroll
    for (int o = 0; o < R; ++o)
#pragma unroll
      for (int off = 32 / G; off < 32; off <<= 1)
#pragma unroll
        for (int u = 0; u < EV; ++u) acc[o].v[u] = add_s(acc[o].v[u], shfl_xor_s(acc[o].v[u], off));
  }
}

// qlist_row dispatched on the block row's size r (1 <= r <= kPipeMaxBs).
template <typename T, int EV, int G = 1>
__device__ __forceinline__ void qlist_row_r(int r, const unsigned short* ql, int nq, const T* vr,
                                            const unsigned char* xl, PipeLane<T, EV> (&acc)[kPipeMaxBs],
                                            int grp = 0) {
  switch (r) {
    case 1: qlist_row<T, EV, 1, G>(ql, nq, vr, xl, acc, grp); break;
    case 2: qlist_row<T, EV, 2, G>(ql, nq, vr, xl, acc, grp); break;
    case 3: qlist_row<T, EV, 3, G>(ql, nq, vr, xl, acc, grp); break;
    case 4: qlist_row<T, EV, 4, G>(ql, nq, vr, xl, acc, grp); break;
    case 5: qlist_row<T, EV, 5, G>(ql, nq, vr, xl, acc, grp); break;
    case 6: qlist_row<T, EV, 6, G>(ql, nq, vr, xl, acc, grp); break;
    case 7: qlist_row<T, EV, 7, G>(ql, nq, vr, xl, acc, grp); break;
    default: qlist_row<T, EV, 8, G>(ql, nq, vr, xl, acc, grp); break;
  }
}

// Resident CTAs per SM the register allocation is held to: FP32 tiles need
// half the shared memory of FP64 ones, so a third CTA fits when the kernel
// keeps to 80 registers (measured: 503k against 396k moment-vectors/s on the
// 200 x 200 lattice KPM, 64 vectors).
template <typename T> struct TileMinCtas { static constexpr int v = 2; };
template <> struct TileMinCtas<float> { static constexpr int v = 3; };

// Persistent CTAs over the tiles, handed out by a work queue or in a fixed
// stride (the autotuner's choice); warp w multiplies the w-th run of the
// tile's block rows (runs planned for balanced work).  Shared memory:
// barrier | values (vbytes16) | q-list (qbytes16) | X rows.  The next tile's
// record is loaded while this one is multiplied; a warp's first row record
// while the tile's copies are in flight.
template <typename T, int EV, int G = 1>
__global__ void __launch_bounds__(kTileWarps * 32, TileMinCtas<T>::v)
    apply_tile_kernel(ApplyArgs a, const T* __restrict__ vals, const int4* __restrict__ tiles,
                      const int4* __restrict__ ranges, const unsigned short* __restrict__ qidx,
                      const int4* __restrict__ rowinfo, int ntiles, unsigned vbytes16, unsigned qbytes16,
                      int* __restrict__ queue, int part_base, int total) {
  using L = PipeLane<T, EV>;
  constexpr int RB = 32 / G * (int)sizeof(L);  // bytes of one X row (32 / G lanes)
  extern __shared__ __align__(16) unsigned char tile_smem[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int gl = lane % (32 / G), grp = lane / (32 / G);  // lane within its group, the group
  const unsigned bar = smem_addr(tile_smem);
  const T* vs_base = reinterpret_cast<const T*>(tile_smem + 16);
  const unsigned short* qs_base = reinterpret_cast<const unsigned short*>(tile_smem + 16 + vbytes16);
  const unsigned char* xs_base = tile_smem + 16 + vbytes16 + qbytes16;
  const unsigned xs_s = smem_addr(xs_base), vs_s = smem_addr(vs_base), qs_s = smem_addr(qs_base);
  const bool use_p = a.gamma != 0.0, use_d = a.want_dots && a.dotw;
  // tiles come from a work queue (queue != nullptr): the first wave takes
  // tiles blockIdx.x, then every CTA claims the tile after its next one
  // (thread 0, one atomic per tile, published in the parity slot of the
  // iteration at the tile's end) so that the next tile's record is always
  // loaded a tile ahead; without a queue CTA b takes tiles b, b + grid, ...
  // (neighbouring tiles run at the same time and share X strips in L2)
  __shared__ int s_claim[2];
  if (threadIdx.x == 0) {
    mbar_init(bar, 1);
    mbar_init_fence();
    s_claim[1] = blockIdx.x >= ntiles ? ntiles
                 : queue           ? (int)gridDim.x + atomicAdd(queue, 1)
                                   : (int)(blockIdx.x + gridDim.x);
  }
  __syncthreads();
  const T* X = static_cast<const T*>(a.X);
  double d0 = 0.0, d1 = 0.0;
  unsigned phase = 0;
  bool failed = false;
  int4 ra, rb, rc, rq;  // the next tile's record
  if (blockIdx.x < ntiles) {
    ra = tiles[4 * blockIdx.x];
    rb = tiles[4 * blockIdx.x + 1];
    rc = tiles[4 * blockIdx.x + 2];
    rq = tiles[4 * blockIdx.x + 3];
  }
  int nt = s_claim[1];
  for (int tile = blockIdx.x, it = 0; tile < ntiles; ++it) {
    const int4 ta = ra, tb = rb, tc = rc, tq = rq;
    if (nt < ntiles) {
      ra = tiles[4 * nt];
      rb = tiles[4 * nt + 1];
      rc = tiles[4 * nt + 2];
      rq = tiles[4 * nt + 3];
    }
    int claimed = ntiles;  // thread 0: the tile after nt (stored at the tile's end)
    const long long k0 = (static_cast<long long>(tb.y) << 32) | static_cast<unsigned>(tb.x);
    if (threadIdx.x == 0) {
      const unsigned vbytes = (unsigned)tb.z, xbytes = (unsigned)tb.w, obytes = (unsigned)tc.y * RB;
      // the previous tile's shared-memory reads come before these copies
      fence_proxy_async();
      mbar_arm(bar, xbytes + vbytes + (unsigned)tq.y);
      bulk_g2s(qs_s, qidx + tq.x, (unsigned)tq.y, bar);
      for (int g = ta.z; g < ta.w; ++g) {
        const int4 rg = ranges[g];
        bulk_g2s(xs_s + (unsigned)rg.z * RB, X + (long long)rg.x * a.ld, (unsigned)rg.y * RB, bar);
      }
      if (vbytes) bulk_g2s(vs_s, vals + k0, vbytes, bar);
      // the epilogue's streamed operands: have L2 fetch the tile's rows
      if (use_p) bulk_prefetch_l2(static_cast<const T*>(a.Xprev) + (long long)tc.z * a.ld, obytes);
      if (use_d) bulk_prefetch_l2(static_cast<const T*>(a.dotw) + (long long)tc.z * a.ld, obytes);
      // claimed after the copies are on their way; the result is stored
      // only at the tile's end, so the atomic's latency hides behind it
      if (nt < ntiles) claimed = queue ? (int)gridDim.x + atomicAdd(queue, 1) : nt + (int)gridDim.x;
    }
    // this warp's run of block rows [row0, row1)
    auto run_end = [&](int k) {  // end of run k within the tile: byte k of (tq.z, tq.w)
      return (int)((((unsigned)(k < 4 ? tq.z : tq.w)) >> (8 * (k & 3))) & 0xffu);
    };
    const int row0 = ta.x + (warp == 0 ? 0 : run_end(warp - 1));
    const int row1 = ta.x + run_end(warp);
    int4 ri = make_int4(0, 0, 0, 0);  // {q-list entry, q-list length, first value, block size}
    long long y0 = 0;
    if (row0 < row1) {
      ri = rowinfo[row0];
      y0 = a.scal_off[row0];
    }
    // warp 0 waits for the copies (bounded); the other warps wait at the
    // CTA barrier instead of polling, then observe the completed phase once
    // (the acquire of the copied data)
    const bool ok = warp == 0 ? pipe_wait(bar, phase) : true;
    if (!__syncthreads_and(ok)) {
      failed = true;
      break;
    }
    (void)mbar_try_wait(bar, phase);
    phase ^= 1u;
    for (int row = row0; row < row1; ++row) {
      if (row != row0) {
        ri = rowinfo[row];
        y0 = a.scal_off[row];
      }
      const int r = ri.w;
      L acc[kPipeMaxBs];
      qlist_row_r<T, EV, G>(r, qs_base + ri.x, ri.y, vs_base + ri.z, xs_base + (size_t)gl * sizeof(L), acc, grp);
      const int orow = (int)(y0 - tc.z);  // this row's first scalar row within the tile
      double rd0 = 0.0, rd1 = 0.0;
      tile_epilogue<T, EV, RB, G>(a, acc, r, y0, gl, xs_base + (size_t)(tc.x + orow) * RB + (size_t)gl * sizeof(L),
                                  rd0, rd1, grp);
      if (a.want_dots) {
        if (a.row_dots) {
          write_row_dots(a.row_dots, row, rd0, rd1);
        } else {
          d0 += rd0;
          d1 += rd1;
        }
      }
    }
    if (threadIdx.x == 0) s_claim[it & 1] = claimed;
    __syncthreads();  // every warp is done with the tile before the next copies
    tile = nt;
    nt = s_claim[it & 1];
  }
  if (failed && threadIdx.x == 0) {
    atomicOr(&g_pipe_status, 1u);
    // the copies of the tile that timed out may still be in flight
    mbar_wait_bounded(bar, phase);
  }
  // this CTA claims no more tiles: the last CTA out resets the queue
  if (queue && threadIdx.x == 0) {
    __threadfence();
    if (atomicAdd(queue + 1, 1) == (int)gridDim.x - 1) {
      queue[0] = 0;
      queue[1] = 0;
      __threadfence();
    }
  }
  if (a.want_dots && !a.row_dots) grid_reduce2(d0, d1, a.partials, a.counter, a.dots_out, part_base, total);
}
