// dbs_cluster.cu -- core marking, cell union-find, cluster ids, border labels.
//
// Reference path replaced (ryanirl/dbscan-torch v0.2.0, csrc/cuda/dbscan_cuda.cu):
//   k_core_pass1 :199-208, k_core_pass2 :213-245, k_cell_status :250-263,
//   uf_find / uf_find_readonly / uf_unite :277-311, k_uf_init :313-316,
//   k_unite_pairs :318-370, k_uf_flatten :374-378, k_root_flag :383-390,
//   thrust::exclusive_scan :698-701, k_cluster_id_per_cell :392-404,
//   k_core_labels :409-417, k_border_assign :427-470, k_unpermute :475-481.
//
// Core marking runs one thread per query point (the points of cells below
// min_samples, listed by k_cell_prep in sorted order, so a warp's threads are
// mostly points of one cell and share its neighbour row, boxes and candidate
// points). Union-find works on compacted cell-pair lists: one thread per
// candidate pair, one warp per pair over the thread's test budget. Labelling
// runs one thread per border point, then one per sorted point. The
// reference's bounding-box prunes are kept exactly, so every pair the
// reference tests is tested with the same arithmetic and the same verdict.
#include "dbs_internal.cuh"

namespace dbs {

constexpr uint32_t kFull = 0xffffffffu;


// ----------------------------------------------------------------- k_core
// Warp-aggregated append of the lanes with `take` to a work list.
__device__ __forceinline__ void append(uint32_t* list, uint32_t* count, bool take, uint32_t v) {
  const uint32_t m = __ballot_sync(kFull, take);
  if (m == 0) return;
  const uint32_t lane = lane_id();
  uint32_t base = 0;
  if (lane == 0) base = atomicAdd(count, (uint32_t)__popc(m));
  base = __shfl_sync(kFull, base, 0);
  if (take) list[base + __popc(m & lanemask_lt())] = v;
}

// The 24 stencil offsets (off = (dx+2)*5 + (dy+2)) without the centre, the
// nearest cells first: sides, diagonals, (+-2, 0) / (0, +-2), (+-1, +-2) /
// (+-2, +-1), corners.
__constant__ int8_t kNearFirst[24] = {7, 11, 13, 17, 6, 8, 16, 18, 2, 10, 14, 22,
                                      1, 3, 5, 9, 15, 19, 21, 23, 0, 4, 20, 24};

// Neighbour cells whose row entry, box and point range one thread loads
// together before it tests any of them (k_core, k_labels): the loads of a
// group are independent, so a thread waits for one memory latency per group
// instead of three dependent ones (row entry -> box -> point range) per cell.
// Wider groups take more registers, hence fewer resident warps. Runs of up to
// kSmallRun points are bound by their slowest threads' chains of dependent
// loads and take the wide form; larger runs are bound by the loads in flight
// across the GPU and take the narrow one (k_core groups of 2, k_labels one
// cell at a time with its loads in program order). Measured on B200 against
// one cell at a time for both: 1M constant-density points, k_core 19.4 ->
// 15.9 us and k_labels 32.3 -> 18.5 us (groups of 4); 100k blobs, 16.5 ->
// 12.6 and 23.2 -> 13.3 us; 10M points, k_core 76.3 -> 71.0 us (groups of
// 2), while groups of 4 (46 and 58 registers) slowed k_core to 87.7 us and
// k_labels from 111.2 to 150.3 us.
constexpr int kNbGroupSmall = 4;
constexpr int kNbGroupLarge = 2;

// Core flag of every query point, one thread per query. A query counts its
// own cell wholesale (the reference never distance-tests the centre cell,
// :231-233) plus the points within eps of the other 24 stencil cells that
// survive the point-box prune (:235-240), stopping once the count reaches
// ms (k_core_pass2 :213-245). Queries that stay non-core go to the border
// list of k_labels.
template <int kNbGroup>
__global__ void __launch_bounds__(kCellThreads) k_core(Plan p) {
  static_assert((kNgh - 1) % kNbGroup == 0, "groups tile the 24 stencil neighbours");
  const uint32_t qn = p.desc->q_count;
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t base = blockIdx.x * blockDim.x; base < qn; base += stride) {
    const uint32_t t = base + threadIdx.x;
    bool noncore = false;
    uint32_t i = 0;
    if (t < qn) {
      i = p.qlist[t];
      const int32_t c = p.point_cell[i];
      const int32_t st0 = p.cell_start[c], st1 = p.cell_start[c + 1];
      const SegParam sp = p.seg_param[p.cell_seg[c]];
      const int32_t ms = sp.ms;
      const float eps_sq = sp.eps_sq;
      int32_t cnt = st1 - st0;
      const float2 q = p.xy[i];
      const int32_t* row = p.ngh + (int64_t)c * kNgh;
      // Nearest cells first, so the count reaches ms (and stops) sooner; a
      // neighbour cell wholly within eps of q (point_box_max_d2) counts all
      // its points without distance tests. Neither changes the core flag.
      for (int g = 0; g < kNgh - 1 && cnt < ms; g += kNbGroup) {
        int32_t nb[kNbGroup], j0[kNbGroup], j1[kNbGroup];
        float4 bb[kNbGroup];
#pragma unroll
        for (int u = 0; u < kNbGroup; ++u) nb[u] = row[kNearFirst[g + u]];
#pragma unroll
        for (int u = 0; u < kNbGroup; ++u) {
          const int32_t s = max(nb[u], 0);  // cell 0 exists: this cloud has cell c
          bb[u] = p.bbox[s];
          j0[u] = p.cell_start[s];
          j1[u] = p.cell_start[s + 1];
        }
#pragma unroll
        for (int u = 0; u < kNbGroup; ++u) {
          if (nb[u] < 0 || cnt >= ms) continue;
          if (!(point_box_d2(q.x, q.y, bb[u]) <= eps_sq)) continue;
          if (point_box_max_d2(q.x, q.y, bb[u]) <= eps_sq) {
            cnt += j1[u] - j0[u];
            continue;
          }
#pragma unroll 4
          for (int32_t j = j0[u]; j < j1[u]; ++j) {
            const float2 pj = p.xy[j];
            cnt += sq_dist(__fsub_rn(pj.x, q.x), __fsub_rn(pj.y, q.y)) <= eps_sq;
          }
        }
      }
      const bool core = cnt >= ms;
      p.is_core[i] = core ? 1 : 0;
      noncore = !core;
    }
    append(p.blist, &p.desc->b_count, noncore, i);
  }
}

// Cell status (dbscan_cuda.cu:250-263) and union-find initialisation
// (:313-316), one thread per cell.
__global__ void __launch_bounds__(256) k_status(Plan p) {
  const uint32_t C = p.desc->num_cells;
  for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < C; c += gridDim.x * blockDim.x) {
    const int32_t s0 = p.cell_start[c], s1 = p.cell_start[c + 1];
    uint8_t st;
    if (s1 - s0 >= p.seg_param[p.cell_seg[c]].ms) {
      st = 2;
    } else {
      bool any = false, all = true;
      for (int32_t j = s0; j < s1; ++j) {
        const bool k = p.is_core[j] != 0;
        any |= k;
        all &= k;
      }
      st = !any ? 0 : (all ? 2 : 1);
    }
    p.cell_status[c] = st;
    p.uf[c] = (int32_t)c;
  }
}

// ------------------------------------------------------------ union-find
__device__ __forceinline__ int32_t uf_find_ro(const int32_t* uf, int32_t x, Desc* d) {
  const volatile int32_t* vuf = uf;
  for (uint32_t it = 0; it < kFindCap; ++it) {
    const int32_t px = vuf[x];
    if (px == x) return x;
    x = px;
  }
  set_error(d, kErrFind);
  return x;
}

// Union of the sets of cells a and b. The reference (dbscan_cuda.cu:301-311)
// finds both roots and hooks the larger under the smaller; here Rem's
// algorithm with splicing does the same union: walk up from whichever side
// has the larger parent, re-pointing it (compare-and-swap) at the other
// side's smaller parent, until both sides share a parent (already one set) or
// a root is reached and hooked. Every pointer only ever decreases
// (uf[x] <= x), so the root of every component is its smallest cell index,
// exactly as in the reference. Unlike root-to-root hooking, concurrent unions
// of neighbouring sets cannot build long chains: a lattice of thousands of
// sets merged at once (points at exactly eps) otherwise left finds walking
// hundreds of links. A splice moves a subtree into the other endpoint's set;
// the walk then continues from its old parent until that part is joined too,
// so no union is lost.
__device__ __forceinline__ void uf_unite(int32_t* uf, int32_t a, int32_t b, Desc* d) {
  volatile int32_t* vuf = uf;
  int32_t rx = a, ry = b;
  for (uint32_t it = 0; it < kFindCap; ++it) {
    int32_t px = vuf[rx], py = vuf[ry];
    if (px == py) return;
    if (px < py) {
      const int32_t t = rx; rx = ry; ry = t;
      const int32_t u = px; px = py; py = u;
    }
    if (rx == px) {
      if (atomicCAS(&uf[rx], rx, py) == rx) return;  // hook the root rx under py < rx
    } else {
      atomicCAS(&uf[rx], px, py);  // splice: py < px, then continue from px
      rx = px;
    }
  }
  set_error(d, kErrFind);
}

// Is there a core point i of cell c and a core point j of cell nc with
// point_box_d2(i, bbox[nc]) <= eps_sq and d2(i, j) <= eps_sq? (the pair scan
// of dbscan_cuda.cu:353-368, warp-cooperative). Points j farther than eps
// from c's box are skipped as well: with the monotone distance form every
// pair they belong to is farther than eps, so the answer is unchanged.
__device__ __forceinline__ bool pair_scan(const Plan& p, int32_t c0, int32_t c1, int32_t n0,
                                          int32_t n1, float4 bb_c, float4 bb_n, float eps_sq) {
  const uint32_t lane = lane_id();
  // First chunk of nc cached in registers.
  const int32_t j = n0 + (int32_t)lane;
  bool jok = j < n1 && p.is_core[j];
  float2 pjr = make_float2(0.f, 0.f);
  if (jok) {
    pjr = p.xy[j];
    jok = point_box_d2(pjr.x, pjr.y, bb_c) <= eps_sq;
  }
  const bool one_chunk = (n1 - n0) <= 32;
  for (int32_t ib = c0; ib < c1; ib += 32) {
    const int32_t i = ib + (int32_t)lane;
    bool oki = i < c1 && p.is_core[i];
    float2 pi = make_float2(0.f, 0.f);
    if (oki) {
      pi = p.xy[i];
      oki = point_box_d2(pi.x, pi.y, bb_n) <= eps_sq;
    }
    uint32_t cm = __ballot_sync(kFull, oki);
    while (cm) {
      const int q = __ffs(cm) - 1;
      cm &= cm - 1;
      const float qx = __shfl_sync(kFull, pi.x, q), qy = __shfl_sync(kFull, pi.y, q);
      bool hit = jok && sq_dist(__fsub_rn(pjr.x, qx), __fsub_rn(pjr.y, qy)) <= eps_sq;
      if (__any_sync(kFull, hit)) return true;
      if (!one_chunk) {
        for (int32_t jb = n0 + 32; jb < n1; jb += 32) {
          const int32_t jj = jb + (int32_t)lane;
          bool h = false;
          if (jj < n1 && p.is_core[jj]) {
            const float2 pj = p.xy[jj];
            h = point_box_d2(pj.x, pj.y, bb_c) <= eps_sq &&
                sq_dist(__fsub_rn(pj.x, qx), __fsub_rn(pj.y, qy)) <= eps_sq;
          }
          if (__any_sync(kFull, h)) return true;
        }
      }
    }
  }
  return false;
}

// Distance tests one lane may spend on its own cell pair before the pair is
// handed to the whole warp (a dense pair without a close core pair would
// otherwise cost |c| * |nc| serial tests, the reference's k_unite_pairs
// worst case).
constexpr int32_t kPairBudget = 96;

// Stencil offsets (off = (dx+2)*5 + (dy+2)) of the two passes, centre
// excluded: pass 0 the four side neighbours; pass 1 the four diagonal
// neighbours and the outer ring of the 5x5 stencil. A diagonal pair needs
// many tests before a close pair turns up (the close points sit near one
// shared corner), but in dense regions it is nearly always joined already
// through the two side neighbours, so after pass 0 and a flatten it is
// dropped without a scan.
constexpr int kPassOffs = 20;
__constant__ int8_t kRingOffs[2][kPassOffs] = {
    {7, 11, 13, 17, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0},
    {6, 8, 16, 18, 0, 1, 2, 3, 4, 5, 9, 10, 14, 15, 19, 20, 21, 22, 23, 24}};

// Edges of the cell graph, in three compacted steps per pass (pass 0 = side
// neighbours; pass 1 = diagonal and outer neighbours, run after a flatten so
// that most of its pairs are already connected):
//   k_pairs       one thread per core cell: its neighbours nc > c of the
//                 pass that are core cells and pass the box-box prune
//                 (dbscan_cuda.cu:329-351); in pass 1 (after a flatten)
//                 pairs already in one component are dropped.
//                 Survivors go to a pair list.
//   k_pair_scan   one thread per listed pair: i over c's core points passing
//                 the point-box prune against nc, j over nc's core points,
//                 early exit on the first pair within eps (:353-368); found
//                 edges are united (high root hooked under low, :301-311).
//                 Pairs that exhaust kPairBudget tests go to a second list.
//   k_pair_warp   one warp per over-budget pair (pair_scan).
// Whether an edge exists does not depend on the order of the tests, and the
// components (rooted at their smallest cell) do not depend on the order of
// the unions, so the labels are those of the reference.
//
// Loads are issued in independent batches of neighbours: their row entries,
// then their status (and, in pass 1, their root), then the boxes of those
// still in play, so a cell waits for three memory latencies per batch
// instead of up to three per neighbour.
template <int RING>
__global__ void __launch_bounds__(256) k_pairs(Plan p) {
  constexpr int nofs = RING == 0 ? 4 : kPassOffs;
  constexpr int kPairsBatch = RING == 0 ? 4 : 5;  // neighbours whose loads go out together
  static_assert(nofs % kPairsBatch == 0, "batches tile the pass's offsets");
  Desc* d = p.desc;
  const uint32_t C = d->num_cells;
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t base = blockIdx.x * blockDim.x; base < C; base += stride) {
    const uint32_t c = base + threadIdx.x;
    uint32_t mask = 0;  // candidate offsets (bit k = kRingOffs[RING][k])
    const int32_t* row = p.ngh + (int64_t)min(c, C - 1) * kNgh;
    if (c < C && p.cell_status[c] != 0) {
      const float eps_sq = p.seg_param[p.cell_seg[c]].eps_sq;
      const float4 bb_c = p.bbox[c];
      // Pass 1 runs after a flatten: every cell points at its root and no
      // union runs during this kernel, so one load is the find. Pairs
      // already in one component are dropped before their boxes are read
      // (in dense regions most pass-1 neighbours are joined already).
      const int32_t root_c = RING == 1 ? p.uf[c] : 0;  // r = -1 below never equals it
#pragma unroll
      for (int h = 0; h < nofs; h += kPairsBatch) {
        int32_t nb[kPairsBatch];
#pragma unroll
        for (int k = 0; k < kPairsBatch; ++k) nb[k] = row[kRingOffs[RING][h + k]];
        bool any = false;
#pragma unroll
        for (int k = 0; k < kPairsBatch; ++k) any |= nb[k] > (int32_t)c;
        if (!any) continue;  // no neighbour above c in this batch (sparse regions)
        uint32_t m = 0;
#pragma unroll
        for (int k = 0; k < kPairsBatch; ++k) {
          const int32_t s = nb[k] > (int32_t)c ? nb[k] : (int32_t)c;
          const uint8_t st = p.cell_status[s];
          const int32_t r = RING == 1 ? p.uf[s] : -1;
          if (nb[k] > (int32_t)c && st != 0 && r != root_c) m |= 1u << k;
        }
#pragma unroll
        for (int k = 0; k < kPairsBatch; ++k) {
          if (!((m >> k) & 1u)) continue;
          if (!(box_box_d2(bb_c, p.bbox[nb[k]]) <= eps_sq)) m &= ~(1u << k);
        }
        mask |= m << h;
      }
    }
    // Warp-aggregated append of a variable number of pairs per lane.
    const uint32_t cnt = __popc(mask);
    uint32_t x = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(kFull, x, o);
      if (lane_id() >= (uint32_t)o) x += y;
    }
    const uint32_t tot = __shfl_sync(kFull, x, 31);
    uint32_t at = 0;
    if (lane_id() == 31 && tot) {
      at = atomicAdd(&d->p_count, tot);
      if ((uint64_t)at + tot > (uint64_t)p.pair_cap) set_error(d, kErrCapacity);
    }
    at = __shfl_sync(kFull, at, 31) + x - cnt;
#pragma unroll
    for (int k = 0; k < nofs; ++k) {
      if (!((mask >> k) & 1u)) continue;
      if (at < p.pair_cap) p.plist[at] = make_int2((int32_t)c, row[kRingOffs[RING][k]]);
      ++at;
    }
  }
}

__global__ void __launch_bounds__(256) k_pair_scan(Plan p) {
  Desc* d = p.desc;
  const int64_t np = min((int64_t)d->p_count, p.pair_cap);
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t base = (int64_t)blockIdx.x * blockDim.x; base < np; base += stride) {
    const uint32_t t = (uint32_t)(base + threadIdx.x);
    bool deferred = false;
    if ((int64_t)t < np) {
      const int2 pr = p.plist[t];
      const int32_t c = pr.x, nb = pr.y;
      const float eps_sq = p.seg_param[p.cell_seg[c]].eps_sq;
      const float4 bb_n = p.bbox[nb];
      const int32_t c0 = p.cell_start[c], c1 = p.cell_start[c + 1];
      const int32_t n0 = p.cell_start[nb], n1 = p.cell_start[nb + 1];
      bool found = false;
      int32_t budget = kPairBudget;
      for (int32_t i = c0; i < c1 && !found && !deferred; ++i) {
        if (!p.is_core[i]) continue;
        const float2 pi = p.xy[i];
        if (!(point_box_d2(pi.x, pi.y, bb_n) <= eps_sq)) continue;
        for (int32_t j = n0; j < n1; ++j) {
          if (--budget < 0) { deferred = true; break; }
          if (!p.is_core[j]) continue;
          const float2 pj = p.xy[j];
          if (sq_dist(__fsub_rn(pj.x, pi.x), __fsub_rn(pj.y, pi.y)) <= eps_sq) { found = true; break; }
        }
      }
      if (found) uf_unite(p.uf, c, nb, d);
    }
    append(p.dlist, &d->d_count, deferred, t);
  }
}

__global__ void __launch_bounds__(256) k_pair_warp(Plan p) {
  Desc* d = p.desc;
  const int64_t nd = min((int64_t)d->d_count, p.pair_cap);
  const uint32_t lane = lane_id();
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t w = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < nd; w += nwarps) {
    const int2 pr = p.plist[p.dlist[w]];
    const int32_t c = pr.x, nb = pr.y;
    const float eps_sq = p.seg_param[p.cell_seg[c]].eps_sq;
    if (pair_scan(p, p.cell_start[c], p.cell_start[c + 1], p.cell_start[nb], p.cell_start[nb + 1],
                  p.bbox[c], p.bbox[nb], eps_sq) && lane == 0)
      uf_unite(p.uf, c, nb, d);
    __syncwarp();
  }
}

// Point every cell at its current root (read-only walks: a concurrent
// writer of uf[c] only ever stores an ancestor of c, so walks still end at
// the root).
// Between the passes: every cell to its root (so a find in pass 1's pair
// listing is one load), and the pair lists emptied for pass 1 (pass 0 starts
// from the counters k_init cleared; pass 0's k_pair_warp, which reads them,
// has finished when this kernel runs).
__global__ void __launch_bounds__(256) k_flatten(Plan p) {
  Desc* d = p.desc;
  const uint32_t C = d->num_cells;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    d->ring_pairs[0] = d->p_count; d->ring_warp[0] = d->d_count;
    d->p_count = 0; d->d_count = 0;
  }
  for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < C; c += gridDim.x * blockDim.x)
    p.uf[c] = uf_find_ro(p.uf, (int32_t)c, d);
}

// ------------------------------------------------------------------ k_ids
// Flatten every cell to its root (read-only walk, dbscan_cuda.cu:374-378) and
// rank the roots of non-noise components in cell order with a decoupled
// look-back exclusive scan (dbscan_cuda.cu:383-404, 698-701).
//
// A tile is kIdsTile consecutive cells; warp w of the block owns the
// 32 * kIdsItems cells from tile_base + w * 32 * kIdsItems, row k of them
// (cells + k * 32 + lane) in item k of its lanes. Every load and store of the
// uf, cell_status and root_rank arrays is then a whole-warp contiguous access,
// and the rank of a root inside its warp is the popcount of the root-flag
// ballots of the rows before it and of the lanes before it in its row.
__global__ void __launch_bounds__(kScanThreads) k_ids(Plan p) {
  __shared__ uint32_t s_warp[kScanThreads / 32];
  __shared__ uint32_t s_tile;
  __shared__ unsigned long long s_excl;
  Desc* d = p.desc;
  const uint32_t C = d->num_cells;
  const int64_t tiles = ((int64_t)C + kIdsTile - 1) / kIdsTile;
  const uint32_t lane = lane_id(), warp = threadIdx.x >> 5;
  const uint32_t lt = lanemask_lt();
  const int nwarps = blockDim.x >> 5;
  while (true) {
    if (threadIdx.x == 0) s_tile = atomicAdd(&d->ctr[kCtrIds], 1u);
    __syncthreads();
    const int64_t tile = s_tile;
    if (tile >= tiles) break;
    const int64_t c0 = tile * kIdsTile + (int64_t)warp * 32 * kIdsItems + lane;
    // Roots of the lane's cells, the walks advanced in lockstep: each round
    // issues one independent load per unfinished walk instead of finishing
    // one walk before starting the next.
    int32_t r[kIdsItems];
    uint32_t open = 0;
#pragma unroll
    for (int k = 0; k < kIdsItems; ++k) {
      const int64_t c = c0 + k * 32;
      r[k] = c < C ? p.uf[c] : (int32_t)c;
      if (c < C && r[k] != (int32_t)c) open |= 1u << k;
    }
    for (uint32_t it = 0; open && it < kFindCap; ++it) {
      int32_t nx[kIdsItems];
#pragma unroll
      for (int k = 0; k < kIdsItems; ++k) nx[k] = (open >> k) & 1u ? p.uf[r[k]] : r[k];
#pragma unroll
      for (int k = 0; k < kIdsItems; ++k) {
        if (nx[k] == r[k]) open &= ~(1u << k);
        r[k] = nx[k];
      }
    }
    if (open) set_error(d, kErrFind);
    uint32_t ball[kIdsItems];
    uint32_t cnt = 0;
#pragma unroll
    for (int k = 0; k < kIdsItems; ++k) {
      const int64_t c = c0 + k * 32;
      bool f = false;
      if (c < C) {
        p.uf[c] = r[k];
        f = r[k] == (int32_t)c && p.cell_status[c] != 0;
      }
      ball[k] = __ballot_sync(kFull, f);
      cnt += __popc(ball[k]);
    }
    if (lane == 0) s_warp[warp] = cnt;
    __syncthreads();
    if (warp == 0) {  // the whole warp walks the look-back
      uint32_t run = 0;
      if (lane == 0)
        for (int wi = 0; wi < nwarps; ++wi) { const uint32_t t = s_warp[wi]; s_warp[wi] = run; run += t; }
      run = __shfl_sync(kFull, run, 0);
      unsigned long long* my = p.ids_status + tile;
      unsigned long long excl = 0;
      if (tile == 0) {
        if (lane == 0) st_relaxed(my, kFlagInc | run);
      } else {
        if (lane == 0) st_relaxed(my, kFlagAgg | run);
        excl = lookback_warp(p.ids_status, tile, 1, d);
        if (lane == 0) st_relaxed(my, kFlagInc | (excl + run));
      }
      if (lane == 0) s_excl = excl;
    }
    __syncthreads();
    uint32_t rnk = (uint32_t)s_excl + s_warp[warp];
#pragma unroll
    for (int k = 0; k < kIdsItems; ++k) {
      const int64_t c = c0 + k * 32;
      if (c < C) p.root_rank[c] = (int32_t)(rnk + __popc(ball[k] & lt));
      rnk += __popc(ball[k]);
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------- k_cid
// Cluster id of every cell: the rank of its root among its cloud's roots
// (k_cluster_id_per_cell, dbscan_cuda.cu:392-404), -1 for cells without a
// core point.
__global__ void __launch_bounds__(256) k_cid(Plan p) {
  const uint32_t C = p.desc->num_cells;
  for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < C; c += gridDim.x * blockDim.x) {
    int32_t id = -1;
    if (p.cell_status[c] != 0)
      id = p.root_rank[p.uf[c]] - p.root_rank[p.seg_info[p.cell_seg[c]].cell_begin];
    p.cid[c] = id;
  }
}

// --------------------------------------------------------------- k_labels
// Final labels, written straight to input order (k_core_labels :409-417,
// k_border_assign :427-470, k_unpermute :475-481). Items [0, b_count) are
// the non-core points of the border list: each takes the cluster of the
// core point within eps that minimises (d2, input index) over the 25
// stencil cells with a core point, pruned by the point-box test, or -1.
// Items after that are all sorted points; core ones take their cell's id.
// Item order: with labels that fit L2 (n <= kCoreFirstPoints, 64 MB), the
// border items go first so their uneven scans overlap the core items of
// other warps (121 us against 136 us at 10M points); with more points the
// core items go first, so the whole grid sweeps the sorted points -- and the
// input-order label writes of the clouds there -- together instead of
// scattering them over the whole label array (3.5 ms against 7.6 ms for a
// 151M-point, 4,096-cloud batch). With kGrouped (runs of up to kSmallRun
// points) a border point loads the row entries, status, boxes and point
// ranges of kNbGroupSmall neighbour cells together, and its core flag and
// coordinates of each candidate together.

template <bool kGrouped>
__global__ void __launch_bounds__(kCellThreads) k_labels(Plan p) {
  const int64_t n = p.n;
  const int64_t bn = p.desc->b_count;
  const int64_t total = bn + n;
  const bool core_first = n > kCoreFirstPoints;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    int64_t i;
    int32_t lab;
    const int64_t bt = core_first ? t - n : t;  // index into the border list
    if (bt >= 0 && bt < bn) {
      i = p.blist[bt];
      const int32_t c = p.point_cell[i];
      const float eps_sq = p.seg_param[p.cell_seg[c]].eps_sq;
      const float2 q = p.xy[i];
      const int32_t* row = p.ngh + (int64_t)c * kNgh;
      unsigned long long best = ~0ull;
      int32_t best_nb = -1;
      float best_d2 = eps_sq;  // no candidate beyond this (eps, then the best so far)
      // Centre cell, then nearest cells first. A cell whose box is farther
      // than the best d2 found so far cannot hold a smaller (d2, index) key:
      // its points are all strictly farther (point_box_d2 is a lower bound of
      // their rounded d2). A box at exactly the best d2 is still scanned, for
      // a tie with a smaller index.
      auto scan_cell = [&](int32_t nb, uint8_t st, float4 bb, int32_t j0, int32_t j1) {
        if (nb < 0 || st == 0) return;
        if (!(point_box_d2(q.x, q.y, bb) <= best_d2)) return;
#pragma unroll 4
        for (int32_t j = j0; j < j1; ++j) {
          const uint8_t cj = p.is_core[j];
          const float2 pj = p.xy[j];
          const float d2 = sq_dist(__fsub_rn(pj.x, q.x), __fsub_rn(pj.y, q.y));
          if (cj && d2 <= eps_sq) {
            // d2 >= +0 and not NaN here, so its bits order like its value.
            const unsigned long long key = ((unsigned long long)__float_as_uint(d2) << 32) | p.perm[j];
            if (key < best) { best = key; best_nb = nb; best_d2 = d2; }
          }
        }
      };
      if constexpr (kGrouped) {
        constexpr int G = kNbGroupSmall;
        scan_cell(c, p.cell_status[c], p.bbox[c], p.cell_start[c], p.cell_start[c + 1]);
        for (int g = 0; g < kNgh - 1; g += G) {
          int32_t nb[G], j0[G], j1[G];
          uint8_t st[G];
          float4 bb[G];
#pragma unroll
          for (int u = 0; u < G; ++u) nb[u] = row[kNearFirst[g + u]];
#pragma unroll
          for (int u = 0; u < G; ++u) {
            const int32_t s = max(nb[u], 0);  // cell 0 exists: this cloud has cell c
            st[u] = p.cell_status[s];
            bb[u] = p.bbox[s];
            j0[u] = p.cell_start[s];
            j1[u] = p.cell_start[s + 1];
          }
#pragma unroll
          for (int u = 0; u < G; ++u) scan_cell(nb[u], st[u], bb[u], j0[u], j1[u]);
        }
      } else {
        for (int o = -1; o < kNgh - 1; ++o) {
          const int32_t nb = row[o < 0 ? 12 : kNearFirst[o]];
          if (nb < 0 || p.cell_status[nb] == 0) continue;
          if (!(point_box_d2(q.x, q.y, p.bbox[nb]) <= best_d2)) continue;
          const int32_t j1 = p.cell_start[nb + 1];
          for (int32_t j = p.cell_start[nb]; j < j1; ++j) {
            if (!p.is_core[j]) continue;
            const float2 pj = p.xy[j];
            const float d2 = sq_dist(__fsub_rn(pj.x, q.x), __fsub_rn(pj.y, q.y));
            if (d2 <= eps_sq) {
              const unsigned long long key = ((unsigned long long)__float_as_uint(d2) << 32) | p.perm[j];
              if (key < best) { best = key; best_nb = nb; best_d2 = d2; }
            }
          }
        }
      }
      lab = best_nb < 0 ? -1 : p.cid[best_nb];
    } else {
      // Core flag, cell and destination loaded together (nearly every point
      // here is core), so the label waits for two memory latencies, not four.
      i = core_first ? t : t - bn;
      const uint8_t core = p.is_core[i];
      const int32_t cell = p.point_cell[i];
      const uint32_t dst = p.perm[i];
      if (!core) continue;
      p.labels[dst] = p.cid[cell];
      continue;
    }
    p.labels[p.perm[i]] = lab;
  }
}

// ------------------------------------------------------------- launchers
cudaError_t launch_core(const Plan& p, cudaStream_t s) {
  if (p.n <= kSmallRun)
    k_core<kNbGroupSmall><<<p.num_sms * p.bps[kTuneCore], kCellThreads, 0, s>>>(p);
  else
    k_core<kNbGroupLarge><<<p.num_sms * p.bps[kTuneCore], kCellThreads, 0, s>>>(p);
  k_status<<<p.num_sms * 8, 256, 0, s>>>(p);
  return cudaGetLastError();
}

cudaError_t launch_union(const Plan& p, cudaStream_t s) {
  for (int ring = 0; ring < 2; ++ring) {
    if (ring == 1) k_flatten<<<p.num_sms * 8, 256, 0, s>>>(p);
    if (ring == 0)
      k_pairs<0><<<p.num_sms * p.bps[kTunePairs], 256, 0, s>>>(p);
    else
      k_pairs<1><<<p.num_sms * p.bps[kTunePairs], 256, 0, s>>>(p);
    k_pair_scan<<<p.num_sms * p.bps[kTunePairScan], 256, 0, s>>>(p);
    k_pair_warp<<<p.num_sms * 8, 256, 0, s>>>(p);
  }
  return cudaGetLastError();
}

cudaError_t launch_ids(const Plan& p, cudaStream_t s) {
  k_ids<<<p.num_sms * 4, kScanThreads, 0, s>>>(p);
  return cudaGetLastError();
}

cudaError_t launch_labels(const Plan& p, cudaStream_t s) {
  k_cid<<<p.num_sms * 4, 256, 0, s>>>(p);
  if (p.n <= kSmallRun)
    k_labels<true><<<p.num_sms * p.bps[kTuneLabels], kCellThreads, 0, s>>>(p);
  else
    k_labels<false><<<p.num_sms * p.bps[kTuneLabels], kCellThreads, 0, s>>>(p);
  return cudaGetLastError();
}

}  // namespace dbs
