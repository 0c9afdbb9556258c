// dbs_cells.cu -- run-length cells, per-cell bounding boxes and neighbour table.
//
// Reference path replaced (ryanirl/dbscan-torch v0.2.0, csrc/cuda/dbscan_cuda.cu):
//   k_boundary_flags :84-89, thrust::inclusive_scan :606-609, the host read of
//   num_cells :612-617 (removed: the count stays on the device),
//   k_point_cell_from_scan :95-101, k_extract_cell_start :106-120,
//   k_cell_bbox :162-177, binsearch_cell / k_build_ngh :125-150.
//
// k_rle turns the sorted keys into cells with one decoupled look-back scan of
// the boundary flags (4096 keys per tile). Cells keep the reference's order
// (ascending unsigned key), so cell indices are the reference's. Dense clouds
// also record each cell in a dense map indexed by the compacted key, so
// neighbour lookup is one load instead of a binary search.
//
// k_cell_prep gives each cell one lane: it folds the bounding box of the
// cell's points and resolves the 25 offsets of the 5x5 stencil in the
// reference's order (off = (dx+2)*5 + (dy+2)); the warp then walks its cells'
// contiguous points to record each point's cell and class (core wholesale,
// or a query for k_core; k_core_pass1 :199-208).
#include "dbs_internal.cuh"

namespace dbs {

// ------------------------------------------------------------------ k_rle
template <typename K>
__device__ __forceinline__ void rle_body(const Plan& p, K* s_keys, uint32_t* s_warp,
                                         uint32_t* s_tile, unsigned long long* s_excl) {
  Desc* d = p.desc;
  const int64_t n = p.n;
  const K* keys = reinterpret_cast<const K*>(p.keys[d->npasses & 1]);
  const uint32_t lane = lane_id(), warp = threadIdx.x >> 5;
  const int nwarps = blockDim.x >> 5;
  while (true) {
    if (threadIdx.x == 0) *s_tile = atomicAdd(&d->ctr[kCtrRle], 1u);
    __syncthreads();
    const int64_t tile = *s_tile;
    if (tile >= p.scan_tiles) break;
    const int64_t base = tile * kScanTile;
    const int32_t valid = (int32_t)min((int64_t)kScanTile, n - base);
    // Coalesced load into shared memory (a thread's loads in flight in two
    // rounds of kScanItems / 2), then blocked reads.
#pragma unroll 1
    for (int r = 0; r < 2; ++r) {
      constexpr int kHalf = kScanItems / 2;
      K kv[kHalf];
#pragma unroll
      for (int k = 0; k < kHalf; ++k) {
        const int32_t j = threadIdx.x + (r * kHalf + k) * kScanThreads;
        if (j < valid) kv[k] = keys[base + j];
      }
#pragma unroll
      for (int k = 0; k < kHalf; ++k) {
        const int32_t j = threadIdx.x + (r * kHalf + k) * kScanThreads;
        if (j < valid) s_keys[j + 1] = kv[k];
      }
    }
    if (threadIdx.x == 0) s_keys[0] = base > 0 ? keys[base - 1] : (K)0;
    __syncthreads();
    const int32_t j0 = threadIdx.x * kScanItems;
    uint32_t flags = 0;
    uint32_t cnt = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
      const int32_t j = j0 + k;
      if (j < valid) {
        const bool f = (base + j == 0) || (s_keys[j + 1] != s_keys[j]);
        flags |= (uint32_t)f << k;
        cnt += f;
      }
    }
    // Block exclusive scan of per-thread counts.
    uint32_t x = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= (uint32_t)o) x += y;
    }
    if (lane == 31) s_warp[warp] = x;
    __syncthreads();
    if (warp == 0) {  // the whole warp walks the look-back
      uint32_t run = 0;
      if (lane == 0)
        for (int w = 0; w < nwarps; ++w) { const uint32_t t = s_warp[w]; s_warp[w] = run; run += t; }
      run = __shfl_sync(0xffffffffu, run, 0);
      unsigned long long* my = p.rle_status + tile;
      unsigned long long excl = 0;
      if (tile == 0) {
        if (lane == 0) st_relaxed(my, kFlagInc | run);
      } else {
        if (lane == 0) st_relaxed(my, kFlagAgg | run);
        excl = lookback_warp(p.rle_status, tile, 1, d);
        if (lane == 0) st_relaxed(my, kFlagInc | (excl + run));
      }
      if (lane == 0) *s_excl = excl;
      if (lane == 0 && base + valid == n) {
        uint32_t total = (uint32_t)(excl + run);
        if ((int64_t)total > n) total = (uint32_t)n;  // only after a failed look-back
        d->num_cells = total;
        p.cell_start[total] = (int32_t)n;
      }
    }
    __syncthreads();
    // c: cells started before this thread's first item.
    uint32_t c = (uint32_t)*s_excl + s_warp[warp] + x - cnt;
    int32_t seg = flags ? seg_of(p, base + j0) : 0;
#pragma unroll 1
    for (int k = 0; k < kScanItems && j0 + k < valid; ++k) {
      const int64_t i = base + j0 + k;
      if ((flags >> k) & 1u) {
        const uint64_t key = (uint64_t)s_keys[j0 + k + 1];
        while (i >= p.seg_off[seg + 1]) ++seg;
        if ((int64_t)c < n) {  // (c >= n only after a failed look-back)
          p.cell_start[c] = (int32_t)i;
          p.cell_key[c] = key;
          p.cell_seg[c] = seg;
          if (i == p.seg_off[seg]) p.seg_info[seg].cell_begin = (int32_t)c;
          const int64_t mb = p.seg_info[seg].map_base;
          if (mb >= 0) p.cell_map[mb + (int64_t)(key - p.seg_info[seg].base)] = (int32_t)c;
        }
        ++c;
      }
    }
    // The reference's k_gather_xy for this thread's items: every perm load,
    // then every coordinate load, in flight together.
    {
      uint32_t src[kScanItems];
#pragma unroll
      for (int k = 0; k < kScanItems; ++k)
        src[k] = j0 + k < valid ? p.perm[base + j0 + k] : 0u;
      float2 v[kScanItems];
#pragma unroll
      for (int k = 0; k < kScanItems; ++k)
        if (j0 + k < valid) v[k] = p.X[src[k]];
#pragma unroll
      for (int k = 0; k < kScanItems; ++k)
        if (j0 + k < valid) p.xy[base + j0 + k] = v[k];
    }
    __syncthreads();
  }
}

__global__ void __launch_bounds__(kScanThreads) k_rle(Plan p) {
  __shared__ __align__(16) unsigned char s_raw[sizeof(uint64_t) * (kScanTile + 1)];
  __shared__ uint32_t s_warp[kScanThreads / 32];
  __shared__ uint32_t s_tile;
  __shared__ unsigned long long s_excl;
  if (p.desc->dense_sort) return;  // cells came from the counting sort
  if (p.desc->key64)
    rle_body<uint64_t>(p, reinterpret_cast<uint64_t*>(s_raw), s_warp, &s_tile, &s_excl);
  else
    rle_body<uint32_t>(p, reinterpret_cast<uint32_t*>(s_raw), s_warp, &s_tile, &s_excl);
}

// ------------------------------------------------------------ k_cell_prep
// First index in [lo, hi) of the sorted cell keys whose key is >= target.
__device__ __forceinline__ int64_t key_lower_bound(const uint64_t* keys, int64_t lo, int64_t hi,
                                                   uint64_t target) {
  while (lo < hi) {
    const int64_t mid = (lo + hi) >> 1;
    if (keys[mid] < target) lo = mid + 1; else hi = mid;
  }
  return lo;
}

constexpr int32_t kBigCell = 64;  // cells above this size reduce their box per warp

// Box of a cell holding a point with a NaN coordinate (nan_box). fminf/fmaxf skip NaN,
// so the folded box would leave that point out; the infinite box keeps every
// prune sound (nothing is pruned against it) and turns off the whole-cell
// shortcut of k_core, which would otherwise count the NaN point. No label
// changes: a NaN point is within eps of nothing.
__device__ __forceinline__ float4 nan_box() { return make_float4(-INFINITY, INFINITY, -INFINITY, INFINITY); }

// Warp-aggregated append of the lanes with `take` to a work list.
__device__ __forceinline__ void append_list(uint32_t* list, uint32_t* count, bool take, uint32_t v) {
  const uint32_t m = __ballot_sync(0xffffffffu, take);
  if (m == 0) return;
  uint32_t base = 0;
  if (lane_id() == 0) base = atomicAdd(count, (uint32_t)__popc(m));
  base = __shfl_sync(0xffffffffu, base, 0);
  if (take) list[base + __popc(m & lanemask_lt())] = v;
}

// One warp per 32 consecutive cells (lane = cell):
//   - bounding box of each cell's points (cells above kBigCell points get
//     theirs from the whole warp; cells above kHugeCell from k_huge_bbox);
//   - the warp's cells own one contiguous range of sorted points: each point
//     gets its cell, and its class (k_core_pass1, dbscan_cuda.cu:199-208): a
//     point of a cell with >= ms points is core wholesale, any other point
//     goes to the query list of k_core. Point-parallel, so the stores are
//     coalesced;
//   - the 25-entry neighbour row of each cell, staged in shared memory and
//     written as one contiguous block per warp.
//
// LPC lanes per cell (32 / LPC cells per warp): with LPC > 1 (runs of up to
// kSmallRun points) the lanes of a cell split its box fold and its five
// neighbour columns, so a small cloud has LPC times as many warps of work.
// A 1M-point cloud has about 64k cells: 2,016 warps of 32 cells for 148
// SMs left 9.7 warps per SM active.
template <int LPC>
__global__ void __launch_bounds__(kCellThreads, 5) k_cell_prep(Plan p) {
  static_assert(LPC == 1 || LPC == 2 || LPC == 4, "lanes per cell");
  constexpr int CPW = 32 / LPC;  // cells per warp
  __shared__ int32_t s_row[kCellThreads / 32][CPW * kNgh];
  const uint32_t full = 0xffffffffu;
  const uint32_t lane = lane_id();
  const uint32_t sub = lane % LPC;   // this lane's part of its cell
  const uint32_t cl = lane / LPC;    // this lane's cell within the warp
  const int lead = (int)(lane - sub);  // first lane of the cell
  int32_t* srow = s_row[threadIdx.x >> 5];
  const uint32_t C = p.desc->num_cells;
  const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t wbase = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * CPW; wbase < C;
       wbase += warps * CPW) {
    const uint32_t c = wbase + cl;
    const bool valid = c < C;
    int32_t s0 = INT32_MAX, s1 = INT32_MAX, seg = 0;
    if (valid) { s0 = p.cell_start[c]; s1 = p.cell_start[c + 1]; seg = p.cell_seg[c]; }
    const bool big = valid && (s1 - s0) > kBigCell;
    const bool huge = big && (s1 - s0) > kHugeCell;
    const bool dense = valid && (s1 - s0) >= p.seg_param[seg].ms;
    if constexpr (LPC > 1) {
      // Each lane of the cell folds every LPC-th point (fminf/fmaxf flush
      // subnormals, as the reference's fold does), then the lanes combine.
      const bool fold = valid && !big;
      float4 b = make_float4(INFINITY, -INFINITY, INFINITY, -INFINITY);
      bool nan = false;
      if (fold) {
        for (int32_t i = s0 + (int32_t)sub; i < s1; i += LPC) {
          const float2 v = p.xy[i];
          nan |= isnan(v.x) || isnan(v.y);
          b.x = fminf(b.x, v.x); b.y = fmaxf(b.y, v.x);
          b.z = fminf(b.z, v.y); b.w = fmaxf(b.w, v.y);
        }
      }
#pragma unroll
      for (int o = 1; o < LPC; o <<= 1) {
        b.x = fminf(b.x, __shfl_xor_sync(full, b.x, o));
        b.y = fmaxf(b.y, __shfl_xor_sync(full, b.y, o));
        b.z = fminf(b.z, __shfl_xor_sync(full, b.z, o));
        b.w = fmaxf(b.w, __shfl_xor_sync(full, b.w, o));
        nan |= __shfl_xor_sync(full, nan ? 1 : 0, o) != 0;
      }
      if (fold && sub == 0) {
        if (s1 - s0 == 1) {  // raw coordinates, as below
          const float2 v = p.xy[s0];
          b = make_float4(v.x, v.x, v.y, v.y);
        }
        p.bbox[c] = nan ? nan_box() : b;
      }
    } else if (valid && !big) {
      // Fold the box. A one-point cell keeps its raw coordinates: the
      // reference seeds the fold with xs[s] and flushes subnormals only
      // through fminf/fmaxf.
      float2 v = p.xy[s0];
      float4 b = make_float4(v.x, v.x, v.y, v.y);
      bool nan = isnan(v.x) || isnan(v.y);
      if (s1 - s0 > 1) {
        b = make_float4(fminf(v.x, INFINITY), fmaxf(v.x, -INFINITY), fminf(v.y, INFINITY),
                        fmaxf(v.y, -INFINITY));
        for (int32_t i = s0 + 1; i < s1; ++i) {
          v = p.xy[i];
          nan |= isnan(v.x) || isnan(v.y);
          b.x = fminf(b.x, v.x); b.y = fmaxf(b.y, v.x);
          b.z = fminf(b.z, v.y); b.w = fmaxf(b.w, v.y);
        }
      }
      p.bbox[c] = nan ? nan_box() : b;
    }
    if (huge && sub == 0) {
      // Registered for k_huge_bbox: one entry, ceil(size / kHugeChunk) chunks.
      const unsigned long long nch = (unsigned long long)((s1 - s0 + kHugeChunk - 1) / kHugeChunk);
      const unsigned long long old = atomicAdd(&p.desc->big_packed, (1ull << 40) + nch);
      const unsigned long long e = old >> 40;
      if ((int64_t)e < p.big_cap) {
        p.big_cell[e] = (int32_t)c;
        p.big_base[e] = old & ((1ull << 40) - 1);
        p.big_done[e] = 0;
      }
    }
    uint32_t bm = __ballot_sync(full, big && !huge && sub == 0);
    while (bm) {
      const int l = __ffs(bm) - 1;
      bm &= bm - 1;
      const int32_t b0 = __shfl_sync(full, s0, l), b1 = __shfl_sync(full, s1, l);
      float xmin = INFINITY, xmax = -INFINITY, ymin = INFINITY, ymax = -INFINITY;
      bool nan = false;
      for (int32_t i = b0 + lane; i < b1; i += 32) {
        const float2 v = p.xy[i];
        nan |= isnan(v.x) || isnan(v.y);
        xmin = fminf(xmin, v.x); xmax = fmaxf(xmax, v.x);
        ymin = fminf(ymin, v.y); ymax = fmaxf(ymax, v.y);
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        xmin = fminf(xmin, __shfl_xor_sync(full, xmin, o));
        xmax = fmaxf(xmax, __shfl_xor_sync(full, xmax, o));
        ymin = fminf(ymin, __shfl_xor_sync(full, ymin, o));
        ymax = fmaxf(ymax, __shfl_xor_sync(full, ymax, o));
      }
      nan = __any_sync(full, nan);
      if ((int)lane == l) p.bbox[c] = nan ? nan_box() : make_float4(xmin, xmax, ymin, ymax);
    }

    // Query slots: a cell below ms points has all its points queried, a
    // dense one none, so one scan of the lanes' query counts and one atomic
    // per 32 cells place every query (in sorted order within the warp's
    // cells), instead of a warp-aggregated atomic per 32 points whose
    // returned base every later step of the walk would wait for.
    const uint32_t nq = (valid && !huge && !dense && sub == 0) ? (uint32_t)(s1 - s0) : 0u;
    uint32_t xq = nq;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(full, xq, o);
      if (lane >= (uint32_t)o) xq += y;
    }
    const uint32_t totq = __shfl_sync(full, xq, 31);
    uint32_t qbase = 0;
    if (lane == 31 && totq) qbase = atomicAdd(&p.desc->q_count, totq);
    uint32_t qfirst = __shfl_sync(full, qbase, 31) + xq - nq;  // this cell's first slot
    if constexpr (LPC > 1) qfirst = __shfl_sync(full, qfirst, lead);

    // Points of the warp's cells, runs of consecutive non-huge cells at a
    // time (huge cells' points are classified by k_huge_bbox).
    uint32_t todo = __ballot_sync(full, valid && !huge);
    while (todo) {
      const int la = __ffs(todo) - 1;
      const uint32_t run = todo >> la;
      const int len = (~run) ? __ffs(~run) - 1 : 32 - la;
      todo &= ~((len >= 32 ? full : ((1u << len) - 1u)) << la);
      const int32_t a = __shfl_sync(full, s0, la), b = __shfl_sync(full, s1, la + len - 1);
      for (int32_t base = a; base < b; base += 32) {
        const int32_t i = base + (int32_t)lane;
        const bool ok = i < b;
        // Lane (cell) of point i: the last lane whose first point is <= i.
        int lo = 0;
#pragma unroll
        for (int step = 16; step > 0; step >>= 1) {
          const int32_t sp = __shfl_sync(full, s0, lo + step);
          if (sp <= i) lo += step;
        }
        const bool dn = __shfl_sync(full, dense, lo);
        const int32_t cs0 = __shfl_sync(full, s0, lo);
        const uint32_t cq = __shfl_sync(full, qfirst, lo);
        if (ok) {
          p.point_cell[i] = (int32_t)(wbase + lo / LPC);
          p.is_core[i] = dn ? 1 : 0;
          if (!dn) p.qlist[cq + (uint32_t)(i - cs0)] = (uint32_t)i;
        }
      }
    }

    // Neighbour row, off = (dx+2)*5 + (dy+2) as in the reference.
    if (valid) {
      const SegInfo g = p.seg_info[seg];  // in registers for the 25 lookups
      // The cell's grid coordinates, from its first point (the key was made
      // from the same coordinates, so no division of the key is needed).
      const float inv_r = p.seg_param[seg].inv_r;
      const float2 v0 = p.xy[s0];
      const int32_t kx = cell_coord(v0.x, inv_r);
      const int32_t ky = cell_coord(v0.y, inv_r);
      uint64_t ngy[5];
#pragma unroll
      for (int dy = 0; dy < 5; ++dy)
        ngy[dy] = compact_axis((int32_t)((uint32_t)ky + (uint32_t)(dy - 2)), g.by, g.py);
      if (g.map_base >= 0 && LPC > 1) {
        // Dense cloud: this lane's map rows (every LPC-th column).
#pragma unroll
        for (int dx = 0; dx < 5; ++dx) {
          if (dx % LPC != (int)sub) continue;
          const uint64_t ngx = compact_axis((int32_t)((uint32_t)kx + (uint32_t)(dx - 2)), g.bx, g.px);
          const int32_t* mrow = p.cell_map + g.map_base + (int64_t)(ngx * g.ys);
#pragma unroll
          for (int dy = 0; dy < 5; ++dy)
            srow[cl * kNgh + dx * 5 + dy] = (ngx != ~0ull && ngy[dy] != ~0ull) ? mrow[ngy[dy]] : -1;
        }
      } else if (g.map_base >= 0) {
        // Dense cloud: five map rows, 25 independent loads.
        int32_t r[25];
#pragma unroll
        for (int dx = 0; dx < 5; ++dx) {
          const uint64_t ngx = compact_axis((int32_t)((uint32_t)kx + (uint32_t)(dx - 2)), g.bx, g.px);
          const int32_t* mrow = p.cell_map + g.map_base + (int64_t)(ngx * g.ys);
#pragma unroll
          for (int dy = 0; dy < 5; ++dy)
            r[dx * 5 + dy] = (ngx != ~0ull && ngy[dy] != ~0ull) ? mrow[ngy[dy]] : -1;
        }
#pragma unroll
        for (int k = 0; k < 25; ++k) srow[cl * kNgh + k] = r[k];
      } else {
        // Sparse cloud: its cells are sorted by key, and the five neighbours
        // of one column (same gx) are the keys base + ngx * ys + ngy[dy].
        // Taken in ascending ngy (a sorting network over the five, invalid
        // coordinates last), consecutive targets of one coordinate class are
        // one key apart, so each is reached from the previous one by a walk
        // of at most one cell; only the first target of a column (and a jump
        // across the class boundary) takes a binary search over the cloud's
        // cells -- 5 searches per cell instead of 25.
        uint64_t sy[5];
        int sd[5];
#pragma unroll
        for (int dy = 0; dy < 5; ++dy) { sy[dy] = ngy[dy]; sd[dy] = dy; }
#define DBS_CS(a, b)                                                      \
  if (sy[b] < sy[a]) {                                                    \
    const uint64_t ty = sy[a]; sy[a] = sy[b]; sy[b] = ty;                 \
    const int td = sd[a]; sd[a] = sd[b]; sd[b] = td;                      \
  }
        DBS_CS(0, 1) DBS_CS(3, 4) DBS_CS(2, 4) DBS_CS(2, 3) DBS_CS(0, 3)
        DBS_CS(0, 2) DBS_CS(1, 4) DBS_CS(1, 3) DBS_CS(1, 2)
#undef DBS_CS
        const int64_t npts = p.seg_off[seg + 1] - p.seg_off[seg];
        const int64_t lo0 = g.cell_begin, hi0 = min((int64_t)C, lo0 + npts);
#pragma unroll
        for (int dx = 0; dx < 5; ++dx) {
          if (dx % LPC != (int)sub) continue;  // another lane's column
          int32_t* out = srow + cl * kNgh + dx * 5;
          const uint64_t ngx = compact_axis((int32_t)((uint32_t)kx + (uint32_t)(dx - 2)), g.bx, g.px);
          if (ngx == ~0ull || sy[0] == ~0ull) {
#pragma unroll
            for (int dy = 0; dy < 5; ++dy) out[dy] = -1;
            continue;
          }
          const uint64_t rowbase = g.base + ngx * g.ys;
          int64_t pos = key_lower_bound(p.cell_key, lo0, hi0, rowbase + sy[0]);
#pragma unroll
          for (int j = 0; j < 5; ++j) {
            if (sy[j] == ~0ull) { out[sd[j]] = -1; continue; }
            const uint64_t t = rowbase + sy[j];
            int steps = 0;
            while (pos < hi0 && p.cell_key[pos] < t) {
              if (++steps > 2) { pos = key_lower_bound(p.cell_key, pos, hi0, t); break; }
              ++pos;
            }
            out[sd[j]] = (pos < hi0 && p.cell_key[pos] == t) ? (int32_t)pos : -1;
          }
        }
      }
    }
    __syncwarp();
    const int32_t rows = (int32_t)min((uint32_t)CPW, C - wbase);
    int32_t* out = p.ngh + (int64_t)wbase * kNgh;
    for (int32_t k = (int32_t)lane; k < rows * kNgh; k += 32) out[k] = srow[k];
    __syncwarp();
  }
}

// Bounding boxes of huge cells (more than kHugeCell points, e.g. a 2M-point
// dense square): every warp of the grid takes kHugeChunk-point chunks of
// any huge cell, reduces the chunk, and the warp that finishes a cell's last
// chunk folds the cell's chunk boxes into bbox[c]. Min and max are
// order-independent, so the box equals the reference's serial fold.
constexpr int kHugeBatch = 8;  // loads a warp of k_huge_bbox keeps in flight

__global__ void __launch_bounds__(256) k_huge_bbox(Plan p) {
  const uint32_t full = 0xffffffffu;
  const uint32_t lane = lane_id();
  Desc* d = p.desc;
  const unsigned long long packed = d->big_packed;
  const int64_t entries = min((int64_t)(packed >> 40), p.big_cap);
  const int64_t chunks = min((int64_t)(packed & ((1ull << 40) - 1)), p.chunk_cap);
  if (entries == 0) return;
  while (true) {
    uint32_t g = 0;
    if (lane == 0) g = atomicAdd(&d->ctr[kCtrBig], 1u);
    g = __shfl_sync(full, g, 0);
    if ((int64_t)g >= chunks) break;
    // Entry owning chunk g: last entry with big_base <= g.
    int64_t lo = 0, hi = entries - 1;
    while (lo < hi) {
      const int64_t mid = (lo + hi + 1) >> 1;
      if (p.big_base[mid] <= g) lo = mid; else hi = mid - 1;
    }
    const int32_t c = p.big_cell[lo];
    const int32_t s0 = p.cell_start[c], s1 = p.cell_start[c + 1];
    const int32_t k = (int32_t)(g - p.big_base[lo]);
    const int32_t a = s0 + k * kHugeChunk, b = min(s1, a + kHugeChunk);
    float xmin = INFINITY, xmax = -INFINITY, ymin = INFINITY, ymax = -INFINITY;
    // The chunk's points also get their cell and class, as k_cell_prep gives
    // every other point (a huge cell is below ms only when ms > kHugeCell).
    const bool dn = (s1 - s0) >= p.seg_param[p.cell_seg[c]].ms;
    // kHugeBatch steps of 32 points have their loads in flight together.
    for (int32_t base0 = a; base0 < b; base0 += 32 * kHugeBatch) {
      float2 v[kHugeBatch];
#pragma unroll
      for (int u = 0; u < kHugeBatch; ++u) {
        const int32_t i = base0 + 32 * u + (int32_t)lane;
        v[u] = i < b ? p.xy[i] : make_float2(0.f, 0.f);
      }
#pragma unroll
      for (int u = 0; u < kHugeBatch; ++u) {
        const int32_t base = base0 + 32 * u;
        if (base >= b) break;  // warp-uniform
        const int32_t i = base + (int32_t)lane;
        const bool ok = i < b;
        if (ok) {
          p.point_cell[i] = c;
          p.is_core[i] = dn ? 1 : 0;
          if (isnan(v[u].x) || isnan(v[u].y)) {  // whole box becomes nan_box()
            xmin = -INFINITY; xmax = INFINITY; ymin = -INFINITY; ymax = INFINITY;
          }
          xmin = fminf(xmin, v[u].x); xmax = fmaxf(xmax, v[u].x);
          ymin = fminf(ymin, v[u].y); ymax = fmaxf(ymax, v[u].y);
        }
        append_list(p.qlist, &d->q_count, ok && !dn, (uint32_t)i);
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      xmin = fminf(xmin, __shfl_xor_sync(full, xmin, o));
      xmax = fmaxf(xmax, __shfl_xor_sync(full, xmax, o));
      ymin = fminf(ymin, __shfl_xor_sync(full, ymin, o));
      ymax = fmaxf(ymax, __shfl_xor_sync(full, ymax, o));
    }
    const int32_t nch = (s1 - s0 + kHugeChunk - 1) / kHugeChunk;
    uint32_t last = 0;
    if (lane == 0) {
      p.big_chunk_box[g] = make_float4(xmin, xmax, ymin, ymax);
      __threadfence();
      last = atomicAdd(&p.big_done[lo], 1u) == (uint32_t)(nch - 1);
    }
    if (__shfl_sync(full, last, 0)) {
      __threadfence();
      const int64_t b0 = (int64_t)p.big_base[lo];
      xmin = INFINITY; xmax = -INFINITY; ymin = INFINITY; ymax = -INFINITY;
      for (int32_t t0 = lane; t0 < nch; t0 += 32 * kHugeBatch) {
        float4 v[kHugeBatch];
#pragma unroll
        for (int u = 0; u < kHugeBatch; ++u) {
          const int32_t t = t0 + 32 * u;
          v[u] = t < nch ? __ldcg(&p.big_chunk_box[b0 + t])
                         : make_float4(INFINITY, -INFINITY, INFINITY, -INFINITY);
        }
#pragma unroll
        for (int u = 0; u < kHugeBatch; ++u) {
          xmin = fminf(xmin, v[u].x); xmax = fmaxf(xmax, v[u].y);
          ymin = fminf(ymin, v[u].z); ymax = fmaxf(ymax, v[u].w);
        }
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        xmin = fminf(xmin, __shfl_xor_sync(full, xmin, o));
        xmax = fmaxf(xmax, __shfl_xor_sync(full, xmax, o));
        ymin = fminf(ymin, __shfl_xor_sync(full, ymin, o));
        ymax = fmaxf(ymax, __shfl_xor_sync(full, ymax, o));
      }
      if (lane == 0) p.bbox[c] = make_float4(xmin, xmax, ymin, ymax);
    }
  }
}

// ------------------------------------------------------------- launchers
cudaError_t launch_rle(const Plan& p, cudaStream_t s) {
  int grid = p.num_sms * 4;
  if (grid > p.scan_tiles) grid = p.scan_tiles > 0 ? p.scan_tiles : 1;
  k_rle<<<grid, kScanThreads, 0, s>>>(p);
  return cudaGetLastError();
}

cudaError_t launch_cell_prep(const Plan& p, cudaStream_t s) {
  if (p.n <= kSmallRun)
    k_cell_prep<4><<<p.num_sms * p.bps[kTuneCellPrep], kCellThreads, 0, s>>>(p);
  else
    k_cell_prep<1><<<p.num_sms * p.bps[kTuneCellPrep], kCellThreads, 0, s>>>(p);
  k_huge_bbox<<<p.num_sms * 4, 256, 0, s>>>(p);
  return cudaGetLastError();
}

}  // namespace dbs
