// Chained row-tiled forward multivector apply.  Included by vbg_apply.cu
// inside namespace vbg, after vbg_tile.cuh (it uses the tiled apply's q-list
// row product and epilogue, mbarrier helpers and bulk copies).
//
// Y = A X (+ the fused epilogue of vbg_cheb_step) for the same multivectors
// and matrices as the tiled apply: warp-wide or half-warp rows (k = 64 or 16
// FP64 / FP32, 32 complex), blocks of at most 8 x 8.
//
// What it changes against the tiled apply:
//  * X reuse across tiles.  For lattice and banded orderings a tile's X rows
//    form a few strips (its own block columns and the neighbouring strips,
//    e.g. the lattice rows above and below).  The host planner orders the
//    tiles into chains whose consecutive tiles share strips -- for a
//    lattice stored row by row, tiles one lattice row apart: a tile's strip
//    "below" is the next tile's own strip and the one after's strip
//    "above" -- and gives each persistent CTA a run of a chain.  The CTA
//    keeps the staged X rows in a shared-memory cache; a tile loads only the
//    strips not already there (extended to what the next tile of the chain
//    needs from the same rows), so X crosses from L2 into shared memory
//    about once per apply instead of three to five times.
//  * No CTA-wide barrier per tile.  One producer warp arms a two-stage ring
//    (a `full` mbarrier per stage counting the bulk-copied bytes of the
//    tile's new X rows and its values; an `empty` mbarrier per stage that
//    every consumer warp arrives on when it is done with the tile) and
//    issues the next tile's copies while the consumer warps multiply the
//    current one.  A consumer warp that finishes its block row early moves
//    on to the next tile as soon as its data is in, and the block row a
//    warp takes rotates from tile to tile, so rows of unequal size (5-row and
//    3-row blocks) even out across tiles instead of stalling every tile.
//  * Xprev and the dot partner are read from global memory in the epilogue
//    (each is read once per apply, staging buys nothing); the producer asks
//    L2 to fetch the tile's rows of them when it arms the tile.
//
// Cache protocol (planned on the host, chain_plan): tile i's new rows go to
// cache rows that neither tile i nor tile i - 1 uses; the producer arms tile
// i only after every consumer warp released tile i - 2 (the `empty` phase of
// its stage), so no copy overwrites rows a warp may still read.  A consumer
// warp has waited for the `full` phase of every earlier tile of its CTA, so
// rows loaded for earlier tiles are visible to it.
//
// Every wait is bounded (kPipeWaitNs); a wait that runs out sets bit 0 of
// g_pipe_status, the warp stops, and the producer waits (bounded) for the
// copies it issued before the CTA leaves.

// consumer warps (block rows per tile): with the producer warp, 16 warps,
// four per SM sub-partition, so each thread may hold 128 registers
constexpr int kChainRowsMax = 15;
// dynamic shared memory of one CTA (one CTA per SM), below the 227 KB a CTA
// may use, leaving room for the static shared memory of the reduction
constexpr size_t kChainSmemBudget = 227 * 1024 - 1024;
constexpr int kChainHeader = 128;  // barriers: full[2], empty[2]
constexpr int kChainMaxRangesPerTile = 64;

__device__ __forceinline__ void mbar_arrive(unsigned bar) {
  asm volatile("mbarrier.arrive.release.cta.shared::cta.b64 _, [%0];\n" ::"r"(bar) : "memory");
}

// Whether applies the tiled kernel takes run its chained variant (when a
// chain plan fits): the library option "apply.chain" (vbg_set_option): 1
// always, 0 never, 2 (default) for 4-byte values only -- measured on the
// 200 x 200 lattice at 64 vectors, the chained tiles are faster in FP32
// (602k against 594k moment-vectors/s) and the balanced unchained tiles in
// FP64 (0.312 against 0.342 ms per step).
static std::atomic<int> g_opt_chain{2};
static bool chain_enabled(int value_bytes) {
  const int v = g_opt_chain.load(std::memory_order_relaxed);
  return v == 1 || (v == 2 && value_bytes == 4);
}

// A chain plan on the host (before upload).  T == 0: no tile height fits.
struct ChainHostPlan {
  int T = 0, ntiles = 0, nctas = 0, cap = 0, stride = 0, qcap = 0;
  int64_t vcap = 0, staged = 0;
  std::vector<int> order, cta_ptr;
  std::vector<int4> tiles, loads, rowinfo;
  std::vector<unsigned short> qidx;  // the q-list in cache rows (as TilePlan::qidx)
};

// Plans the chained tiles of matrix m for X rows of rb bytes and values of
// ves bytes (kernel layout) on the host, for at most nct_max CTAs: tile
// heights tried, chains, per-CTA cache simulation, and a check of the result
// (see below).  Reads the host structure and the spans' host copies.
static void chain_plan_build(const vbg_matrix* m, int rb, int ves, int nct_max, ChainHostPlan& best,
                             std::vector<std::string>* log = nullptr) {
  auto note = [&](int T, const std::string& what) {
    if (log) log->push_back("T=" + std::to_string(T) + ": " + what);
  };
  best = ChainHostPlan();
  const int n = m->n;
  const std::vector<int>& rp = m->h_row_ptr;
  const std::vector<int>& ci = m->h_col_ind;
  const std::vector<int>& bsz = m->h_bsz;
  const std::vector<int64_t>& soff = m->h_scal_off;
  std::vector<int64_t> vrow(n, 0);
  for (int i = 0; i < n; ++i) {
    const int rpad = kernel_layout_rows(bsz[i], ves);
    for (int p = rp[i]; p < rp[i + 1]; ++p) vrow[i] += (int64_t)bsz[ci[p]] * rpad;
  }
  std::vector<int> stamp(n, -1), cols;
  std::vector<int> qstart, qn;
  qlist_layout(m, qstart, qn);
  int tag = 0;
  for (int T : {15, 12, 10, 8}) {
    if (T > kChainRowsMax) continue;
    const int ntiles = (n + T - 1) / T;
    if (ntiles < 1) continue;
    // the X row ranges of every tile: its own block columns and all block
    // columns its blocks touch, merged into runs of consecutive columns
    std::vector<int> rbeg(ntiles + 1, 0);
    std::vector<int2> rg;  // scalar rows [x, y)
    int64_t vmax = 0;
    int qmax = 0;
    bool ok = true;
    for (int t = 0; t < ntiles && ok; ++t) {
      const int t0 = t * T, t1 = std::min(n, t0 + T);
      ++tag;
      cols.clear();
      for (int i = t0; i < t1; ++i)
        if (stamp[i] != tag) {
          stamp[i] = tag;
          cols.push_back(i);
        }
      for (int p = rp[t0]; p < rp[t1]; ++p)
        if (stamp[ci[p]] != tag) {
          stamp[ci[p]] = tag;
          cols.push_back(ci[p]);
        }
      std::sort(cols.begin(), cols.end());
      const size_t first = rg.size();
      for (size_t q = 0; q < cols.size();) {
        size_t e = q + 1;
        while (e < cols.size() && cols[e] == cols[e - 1] + 1) ++e;
        rg.push_back(make_int2((int)soff[cols[q]], (int)soff[cols[e - 1] + 1]));
        q = e;
      }
      ok = rg.size() - first <= (size_t)kChainMaxRangesPerTile;
      rbeg[t + 1] = (int)rg.size();
      int64_t vs = 0;
      for (int i = t0; i < t1; ++i) vs += vrow[i];
      vmax = std::max(vmax, vs);
      qmax = std::max(qmax, qlist_bytes(qstart, t0, t1));
    }
    if (!ok) {
      note(T, "a tile touches more than " + std::to_string(kChainMaxRangesPerTile) + " ranges");
      continue;
    }
    const size_t vbytes16 = tile_vals_bytes(vmax, ves);
    if (kChainHeader + 2 * (vbytes16 + qmax) >= kChainSmemBudget) {
      note(T, "values do not fit");
      continue;
    }
    // cache rows are 16-bit q-list entries
    const int cap = (int)std::min<size_t>((kChainSmemBudget - kChainHeader - 2 * (vbytes16 + qmax)) / rb, 65535);
    // chain stride: the tile that holds the middle of a tile's last strip,
    // the most common offset over all tiles
    int stride = 0;
    {
      std::map<int, int> cnt;
      for (int t = 0; t < ntiles; ++t) {
        if (rbeg[t + 1] == rbeg[t]) continue;
        const int2 g = rg[rbeg[t + 1] - 1];
        const int64_t mid = ((int64_t)g.x + g.y) / 2;
        const int br = (int)(std::upper_bound(soff.begin(), soff.end(), mid) - soff.begin()) - 1;
        const int d = br / T - t;
        if (d > 0) ++cnt[d];
      }
      int bestc = 0;
      for (const auto& kv : cnt)
        if (kv.second > bestc) {
          bestc = kv.second;
          stride = kv.first;
        }
      if (bestc * 2 < ntiles || stride >= ntiles) stride = 0;
    }
    // chained order first, then the natural order (always tried: chains
    // whose strips do not line up with the tiles may not fit the cache)
    for (int attempt = 0; attempt < (stride > 0 ? 2 : 1); ++attempt) {
      const int order_stride = attempt == 0 ? stride : 0;
      ok = true;
      ChainHostPlan c;
      c.T = T;
      c.ntiles = ntiles;
      c.cap = cap;
      c.vcap = vmax;
      c.stride = order_stride;
      c.order.reserve(ntiles);
      if (order_stride > 0) {
        for (int c0 = 0; c0 < order_stride; ++c0)
          for (int t = c0; t < ntiles; t += order_stride) c.order.push_back(t);
      } else {
        for (int t = 0; t < ntiles; ++t) c.order.push_back(t);
      }
      c.nctas = std::max(1, std::min(ntiles, nct_max));
      c.cta_ptr.assign(c.nctas + 1, 0);
      for (int k = 0; k <= c.nctas; ++k) c.cta_ptr[k] = (int)((int64_t)ntiles * k / c.nctas);
      c.qcap = qmax;
      c.tiles.resize(3 * (size_t)ntiles);
      c.qidx.assign(((size_t)qstart[n] + 7) / 8 * 8 + 8, 0);
      c.rowinfo.assign(std::max(n, 1), make_int4(0, 0, 0, 0));
      // per CTA: simulate the cache and record every tile's loads
      struct Res {
        int x0, x1, c0, last;  // X rows [x0, x1) at cache rows [c0, c0 + x1 - x0), last tile that used it
      };
      std::vector<Res> res;
      std::vector<int2> place;  // per range of the current tile: {X row of its resident's start, cache row}
      for (int k = 0; k < c.nctas && ok; ++k) {
        res.clear();
        int head = 0;  // cache row after the latest load
        for (int pos = c.cta_ptr[k]; pos < c.cta_ptr[k + 1] && ok; ++pos) {
          const int i = pos - c.cta_ptr[k];  // local tile index
          const int t = c.order[pos];
          const int g0 = rbeg[t], g1 = rbeg[t + 1];
          place.assign(g1 - g0, make_int2(-1, -1));
          const int lb = (int)c.loads.size();
          // hits: a resident that holds the whole range
          for (int g = g0; g < g1; ++g)
            for (Res& r : res)
              if (r.x0 <= rg[g].x && rg[g].y <= r.x1) {
                r.last = i;
                place[g - g0] = make_int2(r.x0, r.c0);
                break;
              }
          for (int g = g0; g < g1 && ok; ++g) {
            if (place[g - g0].x >= 0) continue;
            // in a chain, extend the load by the rows the next tile needs
            // from the same stretch of X (in the natural order neighbouring
            // tiles overlap by a little on every strip: loads stay exact)
            int x0 = rg[g].x, x1 = rg[g].y;
            if (order_stride > 0 && pos + 1 < c.cta_ptr[k + 1]) {
              const int tn = c.order[pos + 1];
              for (int h = rbeg[tn]; h < rbeg[tn + 1]; ++h)
                if (rg[h].x < x1 && rg[h].y > x0) {
                  x0 = std::min(x0, rg[h].x);
                  x1 = std::max(x1, rg[h].y);
                }
            }
            // Cache rows for the load, handed out like a ring (the rows after
            // the previous load first, then from the start): strips age out
            // of a chain in order, so this keeps the free rows contiguous.
            // Rows that a resident of this or the previous tile holds are
            // never taken.  Without room for the extension, the range alone.
            std::vector<int2> busy;
            for (const Res& r : res)
              if (r.last >= i - 1) busy.push_back(make_int2(r.c0, r.c0 + (r.x1 - r.x0)));
            std::sort(busy.begin(), busy.end(), [](int2 a, int2 b) { return a.x < b.x; });
            auto find_room = [&](int len) -> int {
              int best_at = -1;
              for (int pass = 0; pass < 2 && best_at < 0; ++pass) {
                int at = pass == 0 ? head : 0;
                for (const int2& b : busy) {
                  if (b.y <= at) continue;
                  if (b.x - at >= len) break;
                  at = std::max(at, b.y);
                }
                if (at + len <= cap) best_at = at;
              }
              return best_at;
            };
            int len = x1 - x0;
            int at = len <= cap ? find_room(len) : -1;
            if (at < 0) {
              x0 = rg[g].x;
              x1 = rg[g].y;
              len = x1 - x0;
              at = find_room(len);
            }
            if (at < 0) {
              note(T, "cache full at tile " + std::to_string(t) + " (cta " + std::to_string(k) + ", local " +
                          std::to_string(i) + ", need " + std::to_string(len) + " of " + std::to_string(cap) + ")");
              ok = false;
              break;
            }
            head = at + len >= cap ? 0 : at + len;
            // evict what the new rows overwrite
            res.erase(std::remove_if(res.begin(), res.end(),
                                     [&](const Res& r) { return r.c0 < at + len && at < r.c0 + (r.x1 - r.x0); }),
                      res.end());
            res.push_back({x0, x1, at, i});
            c.loads.push_back(make_int4(x0, len, at, 0));
            c.staged += len;
            place[g - g0] = make_int2(x0, at);
            // later ranges of this tile that the extension covers are hits
            for (int h = g + 1; h < g1; ++h)
              if (place[h - g0].x < 0 && x0 <= rg[h].x && rg[h].y <= x1) place[h - g0] = make_int2(x0, at);
          }
          if (!ok) break;
          // every X row a block row reads, in the cache, via the tile range holding it
          const int t0 = t * T, t1 = std::min(n, t0 + T);
          auto cache_row = [&](int x) {
            int lo = g0, hi = g1 - 1;
            while (lo < hi) {
              const int mid = (lo + hi + 1) / 2;
              if (rg[mid].x <= x) lo = mid;
              else hi = mid - 1;
            }
            return place[lo - g0].y + (x - place[lo - g0].x);
          };
          for (int r = t0; r < t1; ++r) {
            int q = qstart[r];
            for (int p = rp[r]; p < rp[r + 1]; ++p) {
              const int x0 = (int)soff[ci[p]];
              for (int u = 0; u < bsz[ci[p]]; ++u) c.qidx[q++] = (unsigned short)cache_row(x0 + u);
            }
          }
          c.tiles[3 * (size_t)pos] = make_int4(t0, t1, lb, (int)c.loads.size());
          c.tiles[3 * (size_t)pos + 1] = make_int4(0, 0, 0, cache_row((int)soff[t0]));
          c.tiles[3 * (size_t)pos + 2] = make_int4(qlist_base(qstart, t0), qlist_bytes(qstart, t0, t1), 0, 0);
        }
      }
      if (!ok) continue;
      // value offsets: tiles are runs of consecutive rows, whose kernel-layout
      // values are contiguous
      {
        std::vector<int64_t> tstart(ntiles + 1, 0);
        for (int t = 0; t < ntiles; ++t) {
          int64_t vs = 0;
          for (int i = t * T; i < std::min(n, t * T + T); ++i) vs += vrow[i];
          tstart[t + 1] = tstart[t] + vs;
        }
        for (int pos = 0; pos < ntiles; ++pos) {
          const int t = c.order[pos];
          const int64_t k0 = tstart[t];
          int4& b = c.tiles[3 * (size_t)pos + 1];
          b.x = (int)(k0 & 0xffffffff);
          b.y = (int)(k0 >> 32);
          b.z = (int)((tstart[t + 1] - k0) * ves);
          const int t0 = t * T, t1 = std::min(n, t0 + T), qb = qlist_base(qstart, t0);
          int64_t v = 0;
          for (int i = t0; i < t1; ++i) {
            c.rowinfo[i] = make_int4(qstart[i] - qb, qn[i], (int)v, bsz[i]);
            v += vrow[i];
          }
        }
      }
      // Check the plan against its own promises before it is used: every
      // copy stays inside the cache, no two copies of a tile overlap, no copy
      // overwrites rows the previous tile reads, and every X row a tile reads
      // (its q-lists, its own rows) holds that row when the tile runs.
      {
        std::vector<int> src_at(cap, -1), read_by(cap, -1), written_by(cap, -1);
        for (int k = 0; k < c.nctas && ok; ++k) {
          std::fill(src_at.begin(), src_at.end(), -1);
          std::fill(read_by.begin(), read_by.end(), -1);
          std::fill(written_by.begin(), written_by.end(), -1);
          for (int pos = c.cta_ptr[k]; pos < c.cta_ptr[k + 1] && ok; ++pos) {
            const int i = pos - c.cta_ptr[k];
            const int4 ta = c.tiles[3 * (size_t)pos], tv = c.tiles[3 * (size_t)pos + 1];
            for (int g = ta.z; g < ta.w && ok; ++g) {
              const int4 ld = c.loads[g];
              if (ld.y <= 0 || ld.z < 0 || ld.z + ld.y > cap || ld.x < 0 || (int64_t)ld.x + ld.y > m->N) {
                ok = false;
                break;
              }
              for (int q = 0; q < ld.y; ++q) {
                const int row = ld.z + q;
                if (written_by[row] == i || (read_by[row] >= 0 && read_by[row] >= i - 1)) {
                  ok = false;
                  break;
                }
                written_by[row] = i;
                src_at[row] = ld.x + q;
              }
            }
            if (tv.z < 0 || (size_t)tv.z > vbytes16) ok = false;
            auto reads = [&](int crow, int64_t x, int cnt) {
              if (crow < 0 || crow + cnt > cap) return false;
              for (int q = 0; q < cnt; ++q) {
                if (src_at[crow + q] != x + q) return false;
                read_by[crow + q] = i;
              }
              return true;
            };
            for (int r = ta.x; r < ta.y && ok; ++r) {
              int q = qstart[r];
              for (int p = rp[r]; p < rp[r + 1] && ok; ++p) {
                const int x0 = (int)soff[ci[p]];
                for (int u = 0; u < bsz[ci[p]] && ok; ++u) ok = reads(c.qidx[q++], x0 + u, 1);
              }
            }
            if (ok) ok = reads(tv.w, soff[ta.x], (int)(soff[ta.y] - soff[ta.x]));
          }
        }
        if (!ok) {
          note(T, "self-check failed");
          continue;
        }
      }
      note(T, "stride " + std::to_string(c.stride) + ", staged X rows " + std::to_string(c.staged));
      // fewest staged X rows wins; among near ties the taller tile (more warps)
      if (best.T == 0 || c.staged * 100 < best.staged * 97) best = std::move(c);
    }
  }
}

// The chain plan of matrix m for X rows of rb bytes and values of ves bytes,
// planned once per structure and uploaded; *out = nullptr when no tile
// height fits.  Needs the spans.
static int chain_plan(const vbg_matrix* cm, int rb, int ves, cudaStream_t s, ChainPlan** out) {
  auto* m = const_cast<vbg_matrix*>(cm);
  *out = nullptr;
  const auto key = std::make_pair(rb, ves);
  auto found = m->chain_plans.find(key);
  if (found != m->chain_plans.end()) {
    if (found->second->rows > 0) *out = found->second.get();
    return 0;
  }
  VBG_CHECK(m->span_cap > 0 && (int64_t)m->h_span_x.size() == m->nspans, VBG_E_STATE, "chain plan needs the spans");
  int rc = ensure_host_structure(m, s);
  if (rc) return rc;
  ChainHostPlan best;
  chain_plan_build(m, rb, ves, sm_count(), best);
  auto plan = std::make_unique<ChainPlan>();
  if (best.T == 0) {  // remembered as infeasible
    m->chain_plans[key] = std::move(plan);
    return 0;
  }
  plan->rows = best.T;
  plan->ntiles = best.ntiles;
  plan->nctas = best.nctas;
  plan->cap_rows = best.cap;
  plan->vcap = best.vcap;
  plan->stride = best.stride;
  plan->staged_rows = best.staged;
  plan->qcap = best.qcap;
  plan->smem = (int)(kChainHeader + 2 * (tile_vals_bytes(best.vcap, ves) + best.qcap) + (size_t)best.cap * rb);
  if ((rc = plan->tiles.ensure(best.tiles.size() * sizeof(int4), s))) return rc;
  if ((rc = plan->loads.ensure(std::max<size_t>(best.loads.size(), 1) * sizeof(int4), s))) return rc;
  if ((rc = plan->cta_ptr.ensure(best.cta_ptr.size() * sizeof(int), s))) return rc;
  if ((rc = plan->qidx.ensure(best.qidx.size() * sizeof(unsigned short), s))) return rc;
  if ((rc = plan->rowinfo.ensure(best.rowinfo.size() * sizeof(int4), s))) return rc;
  VBG_CUDA(cudaMemcpyAsync(plan->tiles.p, best.tiles.data(), best.tiles.size() * sizeof(int4), cudaMemcpyHostToDevice,
                           s));
  if (!best.loads.empty())
    VBG_CUDA(cudaMemcpyAsync(plan->loads.p, best.loads.data(), best.loads.size() * sizeof(int4),
                             cudaMemcpyHostToDevice, s));
  VBG_CUDA(cudaMemcpyAsync(plan->cta_ptr.p, best.cta_ptr.data(), best.cta_ptr.size() * sizeof(int),
                           cudaMemcpyHostToDevice, s));
  VBG_CUDA(cudaMemcpyAsync(plan->qidx.p, best.qidx.data(), best.qidx.size() * sizeof(unsigned short),
                           cudaMemcpyHostToDevice, s));
  VBG_CUDA(cudaMemcpyAsync(plan->rowinfo.p, best.rowinfo.data(), best.rowinfo.size() * sizeof(int4),
                           cudaMemcpyHostToDevice, s));
  VBG_CUDA(cudaStreamSynchronize(s));  // the host vectors are locals
  *out = plan.get();
  m->chain_plans[key] = std::move(plan);
  return 0;
}

// Persistent CTAs (one per SM) over their runs of tiles; warps [0, trows)
// consume, warp trows produces.  Shared memory: barriers (full[2] at 0,
// empty[2] at 16) | values stage 0 | values stage 1 (vbytes16 each) |
// q-list stage 0 | q-list stage 1 (qbytes16 each) | X cache.
template <typename T, int EV, int G = 1>
__global__ void __launch_bounds__((kChainRowsMax + 1) * 32, 1)
    apply_chain_kernel(ApplyArgs a, const T* __restrict__ vals, const int4* __restrict__ tiles,
                       const int4* __restrict__ loads, const int* __restrict__ cta_ptr,
                       const unsigned short* __restrict__ qidx, const int4* __restrict__ rowinfo, int trows,
                       unsigned vbytes16, unsigned qbytes16, int part_base, int total) {
  using L = PipeLane<T, EV>;
  constexpr int RB = 32 / G * (int)sizeof(L);  // bytes of one X row (32 / G lanes)
  extern __shared__ __align__(128) unsigned char chain_smem[];
  __shared__ volatile int failed;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int gl = lane % (32 / G), grp = lane / (32 / G);  // lane within its group, the group
  const unsigned full0 = smem_addr(chain_smem), empty0 = full0 + 16;
  const unsigned char* vbase0 = chain_smem + kChainHeader;  // stage st at vbase0 + st * vbytes16
  const unsigned char* qbase0 = vbase0 + 2 * (size_t)vbytes16;  // stage st at qbase0 + st * qbytes16
  const unsigned char* xcache = qbase0 + 2 * (size_t)qbytes16;
  if (threadIdx.x == 0) {
    mbar_init(full0, 1);
    mbar_init(full0 + 8, 1);
    mbar_init(empty0, trows);
    mbar_init(empty0 + 8, trows);
    mbar_init_fence();
    failed = 0;
  }
  __syncthreads();
  const int tb0 = cta_ptr[blockIdx.x], nt = cta_ptr[blockIdx.x + 1] - tb0;
  double d0 = 0.0, d1 = 0.0;
  if (warp == trows) {
    // producer: lane 0 arms the tiles in order
    if (lane == 0) {
      const T* X = static_cast<const T*>(a.X);
      const unsigned xc_s = smem_addr(xcache);
      int armed = 0;
      for (int i = 0; i < nt; ++i) {
        const int st = i & 1;
        if (i >= 2 && !mbar_wait_bounded(empty0 + 8 * st, ((i >> 1) - 1) & 1)) {
          failed = 1;
          break;
        }
        if (failed) break;
        const int4 ta = tiles[3 * (tb0 + i)], tv = tiles[3 * (tb0 + i) + 1], tq = tiles[3 * (tb0 + i) + 2];
        unsigned xbytes = 0;
        for (int g = ta.z; g < ta.w; ++g) xbytes += (unsigned)loads[g].y * RB;
        fence_proxy_async();  // consumers' reads of the rows being replaced come first
        mbar_arm(full0 + 8 * st, xbytes + (unsigned)tv.z + (unsigned)tq.y);
        bulk_g2s(smem_addr(qbase0 + st * qbytes16), qidx + tq.x, (unsigned)tq.y, full0 + 8 * st);
        for (int g = ta.z; g < ta.w; ++g) {
          const int4 ld = loads[g];
          bulk_g2s(xc_s + (unsigned)ld.z * RB, X + (long long)ld.x * a.ld, (unsigned)ld.y * RB, full0 + 8 * st);
        }
        if (tv.z) {
          const long long k0 = (static_cast<long long>(tv.y) << 32) | static_cast<unsigned>(tv.x);
          bulk_g2s(smem_addr(vbase0 + st * vbytes16), vals + k0, (unsigned)tv.z, full0 + 8 * st);
        }
        // the epilogue's streamed operands: have L2 fetch the tile's rows
        const long long y0 = a.scal_off[ta.x];
        const unsigned obytes = (unsigned)(a.scal_off[ta.y] - y0) * RB;
        if (a.gamma != 0.0) bulk_prefetch_l2(static_cast<const T*>(a.Xprev) + y0 * a.ld, obytes);
        if (a.want_dots && a.dotw) bulk_prefetch_l2(static_cast<const T*>(a.dotw) + y0 * a.ld, obytes);
        ++armed;
      }
      // the copies of the last tiles may still be in flight
      for (int i = std::max(0, armed - 2); i < armed; ++i) (void)mbar_wait_bounded(full0 + 8 * (i & 1), (i >> 1) & 1);
    }
    __syncwarp();
  } else {
    for (int i = 0; i < nt; ++i) {
      const int st = i & 1;
      const int4 ta = tiles[3 * (tb0 + i)], tv = tiles[3 * (tb0 + i) + 1];
      const int row = ta.x + (warp + i) % trows;  // the block row rotates over the warps from tile to tile
      const bool mine = row < ta.y;
      int4 ri = make_int4(0, 0, 0, 0);  // {q-list entry, q-list length, first value, block size}
      long long y0 = 0;
      if (mine) {  // the row's record before the wait
        ri = rowinfo[row];
        y0 = a.scal_off[row];
      }
      if (!pipe_wait(full0 + 8 * st, (i >> 1) & 1)) {
        failed = 1;
        break;
      }
      if (mine) {
        const int r = ri.w;
        const T* vs_base = reinterpret_cast<const T*>(vbase0 + st * vbytes16);
        const unsigned short* qs_base = reinterpret_cast<const unsigned short*>(qbase0 + st * qbytes16);
        L acc[kPipeMaxBs];
        qlist_row_r<T, EV, G>(r, qs_base + ri.x, ri.y, vs_base + ri.z, xcache + (size_t)gl * sizeof(L), acc, grp);
        // this row's own X rows sit right after the tile's first own row in the cache
        const long long orow = y0 - a.scal_off[ta.x];
        double rd0 = 0.0, rd1 = 0.0;
        tile_epilogue<T, EV, RB, G>(a, acc, r, y0, gl,
                                  xcache + ((size_t)tv.w + (size_t)orow) * RB + (size_t)gl * sizeof(L), rd0, rd1,
                                  grp);
        if (a.want_dots) {
          if (a.row_dots) {
            write_row_dots(a.row_dots, row, rd0, rd1);
          } else {
            d0 += rd0;
            d1 += rd1;
          }
        }
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(empty0 + 8 * st);
    }
  }
  __syncthreads();
  if (failed && threadIdx.x == 0) atomicOr(&g_pipe_status, 1u);
  if (a.want_dots && !a.row_dots) grid_reduce2(d0, d1, a.partials, a.counter, a.dots_out, part_base, total);
}
