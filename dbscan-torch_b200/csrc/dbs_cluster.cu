// dbs_cluster.cu -- core marking, cell union-find, cluster ids, border labels.
//
// Reference path replaced (ryanirl/dbscan-torch v0.2.0, csrc/cuda/dbscan_cuda.cu):
//   k_core_pass1 :199-208, k_core_pass2 :213-245, k_cell_status :250-263,
//   uf_find / uf_find_readonly / uf_unite :277-311, k_uf_init :313-316,
//   k_unite_pairs :318-370, k_uf_flatten :374-378, k_root_flag :383-390,
//   thrust::exclusive_scan :698-701, k_cluster_id_per_cell :392-404,
//   k_core_labels :409-417, k_border_assign :427-470, k_unpermute :475-481.
//
// Every cell-level kernel gives one warp to one cell (cells taken in
// ascending order from an atomic counter). The 5x5 neighbourhood of a cell
// is flattened into one list of candidate points: lanes hold the 24 (or 25)
// neighbour cells, a warp scan of their sizes gives each lane's slice, and
// each step the 32 lanes test 32 candidates against one query point at a
// time with ballots. The per-(query, neighbour-cell) bounding-box prune of
// the reference is kept exactly (a bit mask per query), so every pair the
// reference tests is tested with the same arithmetic and the same verdict.
#include "dbs_internal.cuh"

namespace dbs {

constexpr uint32_t kFull = 0xffffffffu;
constexpr int kWarpsPerBlock = kCellThreads / 32;

__device__ __forceinline__ uint32_t next_cell(uint32_t* ctr) {
  uint32_t c = 0;
  if (lane_id() == 0) c = atomicAdd(ctr, 1u);
  return __shfl_sync(kFull, c, 0);
}

// Smallest lane l with pre[l] > f (pre: inclusive prefix, 32 entries).
__device__ __forceinline__ int slice_of(const int32_t* pre, int32_t f) {
  int lo = 0;
#pragma unroll
  for (int step = 16; step > 0; step >>= 1)
    if (pre[lo + step - 1] <= f) lo += step;
  return lo;
}

// Warp inclusive scan.
__device__ __forceinline__ int32_t warp_incl_scan(int32_t v) {
  const uint32_t lane = lane_id();
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int32_t y = __shfl_up_sync(kFull, v, o);
    if (lane >= (uint32_t)o) v += y;
  }
  return v;
}

// ----------------------------------------------------------------- k_core
// Core flag of every point and the cell status. Cells with >= ms points are
// core wholesale (k_core_pass1). Otherwise each point counts its own cell
// wholesale (the reference never distance-tests the centre cell, :231-233)
// plus the points within eps in the other 24 cells that survive the
// point-box prune (:235-240).
__global__ void __launch_bounds__(kCellThreads) k_core(Plan p) {
  __shared__ int32_t s_pre[kWarpsPerBlock][32];
  __shared__ int32_t s_off[kWarpsPerBlock][32];
  const uint32_t lane = lane_id();
  const uint32_t w = threadIdx.x >> 5;
  const uint32_t C = p.desc->num_cells;
  while (true) {
    const uint32_t c = next_cell(&p.desc->ctr[kCtrCore]);
    if (c >= C) break;
    const int32_t st0 = p.cell_start[c], st1 = p.cell_start[c + 1];
    const int32_t npts = st1 - st0;
    const SegParam sp = p.seg_param[p.cell_seg[c]];
    const int32_t ms = sp.ms;
    const float eps_sq = sp.eps_sq;
    if (lane == 0) p.uf[c] = (int32_t)c;
    if (npts >= ms) {
      for (int32_t i = st0 + lane; i < st1; i += 32) p.is_core[i] = 1;
      if (lane == 0) p.cell_status[c] = 2;
      continue;
    }
    int32_t nb = -1, sz = 0, cs0 = 0;
    float4 bb = make_float4(0.f, 0.f, 0.f, 0.f);
    if (lane < kNgh && lane != 12) {
      nb = p.ngh[(int64_t)c * kNgh + lane];
      if (nb >= 0) {
        cs0 = p.cell_start[nb];
        sz = p.cell_start[nb + 1] - cs0;
        bb = p.bbox[nb];
      }
    }
    bool any_core = false, all_core = true;
    for (int32_t qb = 0; qb < npts; qb += 32) {
      const int32_t nq = min(32, npts - qb);
      float2 q = make_float2(0.f, 0.f);
      if ((int32_t)lane < nq) q = p.xy[st0 + qb + lane];
      // Prune mask per query: bit l set when neighbour cell l is not pruned.
      uint32_t mymask = 0;
      for (int32_t j = 0; j < nq; ++j) {
        const float qx = __shfl_sync(kFull, q.x, j), qy = __shfl_sync(kFull, q.y, j);
        const bool ok = nb >= 0 && point_box_d2(qx, qy, bb) <= eps_sq;
        const uint32_t m = __ballot_sync(kFull, ok);
        if ((int32_t)lane == j) mymask = m;
      }
      const uint32_t U = __reduce_or_sync(kFull, (int32_t)lane < nq ? mymask : 0u);
      const int32_t szU = ((U >> lane) & 1u) ? sz : 0;
      const int32_t pre = warp_incl_scan(szU);
      const int32_t T = __shfl_sync(kFull, pre, 31);
      s_pre[w][lane] = pre;
      s_off[w][lane] = cs0 - (pre - szU);
      __syncwarp();
      int32_t cnt = npts;  // lane j: count of query j
      for (int32_t f0 = 0; f0 < T; f0 += 32) {
        const int32_t f = f0 + (int32_t)lane;
        int l = 0;
        float2 pj = make_float2(0.f, 0.f);
        const bool have = f < T;
        if (have) {
          l = slice_of(s_pre[w], f);
          pj = p.xy[f + s_off[w][l]];
        }
        for (int32_t j = 0; j < nq; ++j) {
          const float qx = __shfl_sync(kFull, q.x, j), qy = __shfl_sync(kFull, q.y, j);
          const uint32_t m = __shfl_sync(kFull, mymask, j);
          const bool ok = have && ((m >> l) & 1u) &&
                          sq_dist(__fsub_rn(pj.x, qx), __fsub_rn(pj.y, qy)) <= eps_sq;
          const uint32_t b = __ballot_sync(kFull, ok);
          if ((int32_t)lane == j) cnt += __popc(b);
        }
        if (__ballot_sync(kFull, (int32_t)lane < nq && cnt < ms) == 0) break;
      }
      const bool core = (int32_t)lane < nq && cnt >= ms;
      if ((int32_t)lane < nq) p.is_core[st0 + qb + lane] = core ? 1 : 0;
      any_core |= __ballot_sync(kFull, core) != 0;
      all_core &= __ballot_sync(kFull, (int32_t)lane < nq && !core) == 0;
      __syncwarp();
    }
    if (lane == 0) p.cell_status[c] = !any_core ? 0 : (all_core ? 2 : 1);
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

// Path-halving find (relaxed writes only redirect to ancestors).
__device__ __forceinline__ int32_t uf_find(int32_t* uf, int32_t x, Desc* d) {
  volatile int32_t* vuf = uf;
  int32_t px = vuf[x];
  for (uint32_t it = 0; it < kFindCap; ++it) {
    if (px == x) return x;
    const int32_t gp = vuf[px];
    vuf[x] = gp;
    x = px;
    px = gp;
  }
  set_error(d, kErrFind);
  return x;
}

// Hook the larger root under the smaller (dbscan_cuda.cu:301-311), so the
// root of every component is its smallest cell index.
__device__ __forceinline__ void uf_unite(int32_t* uf, int32_t a, int32_t b, Desc* d) {
  for (uint32_t it = 0; it < kFindCap; ++it) {
    a = uf_find(uf, a, d);
    b = uf_find(uf, b, d);
    if (a == b) return;
    const int32_t hi = a > b ? a : b, lo = a < b ? a : b;
    if (atomicCAS(&uf[hi], hi, lo) == hi) return;
  }
  set_error(d, kErrFind);
}

// Is there a core point i of cell c and a core point j of cell nc with
// point_box_d2(i, bbox[nc]) <= eps_sq and d2(i, j) <= eps_sq? (the pair scan
// of dbscan_cuda.cu:353-368, warp-cooperative).
__device__ __forceinline__ bool pair_scan(const Plan& p, int32_t c0, int32_t c1, int32_t n0,
                                          int32_t n1, float4 bb_n, float eps_sq) {
  const uint32_t lane = lane_id();
  // First chunk of nc cached in registers.
  const int32_t j = n0 + (int32_t)lane;
  const bool jin = j < n1;
  const bool jcore = jin && p.is_core[j];
  float2 pjr = make_float2(0.f, 0.f);
  if (jcore) pjr = p.xy[j];
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
      bool hit = jcore && sq_dist(__fsub_rn(pjr.x, qx), __fsub_rn(pjr.y, qy)) <= eps_sq;
      if (__any_sync(kFull, hit)) return true;
      if (!one_chunk) {
        for (int32_t jb = n0 + 32; jb < n1; jb += 32) {
          const int32_t jj = jb + (int32_t)lane;
          bool h = false;
          if (jj < n1 && p.is_core[jj]) {
            const float2 pj = p.xy[jj];
            h = sq_dist(__fsub_rn(pj.x, qx), __fsub_rn(pj.y, qy)) <= eps_sq;
          }
          if (__any_sync(kFull, h)) return true;
        }
      }
    }
  }
  return false;
}

// Ring-1 offsets of the 5x5 stencil (|dx|,|dy| <= 1, centre excluded).
constexpr uint32_t kRing1 = (1u << 6) | (1u << 7) | (1u << 8) | (1u << 11) | (1u << 13) |
                            (1u << 16) | (1u << 17) | (1u << 18);

__global__ void __launch_bounds__(kCellThreads) k_union(Plan p) {
  const uint32_t lane = lane_id();
  Desc* d = p.desc;
  const uint32_t C = d->num_cells;
  while (true) {
    const uint32_t c = next_cell(&d->ctr[kCtrUnion]);
    if (c >= C) break;
    if (p.cell_status[c] == 0) continue;
    const float eps_sq = p.seg_param[p.cell_seg[c]].eps_sq;
    int32_t nb = -1;
    bool cand = false;
    if (lane < kNgh && lane != 12) {
      nb = p.ngh[(int64_t)c * kNgh + lane];
      cand = nb > (int32_t)c && p.cell_status[nb] != 0;
    }
    const uint32_t mask = __ballot_sync(kFull, cand);
    if (!mask) continue;
    const float4 bb_c = p.bbox[c];
    const int32_t c0 = p.cell_start[c], c1 = p.cell_start[c + 1];
    // Ring-1 neighbours first: their unions make most ring-2 scans redundant.
    uint32_t order[2] = {mask & kRing1, mask & ~kRing1};
    for (int r = 0; r < 2; ++r) {
      uint32_t m = order[r];
      while (m) {
        const int l = __ffs(m) - 1;
        m &= m - 1;
        const int32_t nc = __shfl_sync(kFull, nb, l);
        int same = 0;
        if (lane == 0) same = uf_find_ro(p.uf, (int32_t)c, d) == uf_find_ro(p.uf, nc, d);
        if (__shfl_sync(kFull, same, 0)) continue;
        const float4 bb_n = p.bbox[nc];
        if (!(box_box_d2(bb_c, bb_n) <= eps_sq)) continue;
        const bool found = pair_scan(p, c0, c1, p.cell_start[nc], p.cell_start[nc + 1], bb_n, eps_sq);
        if (found && lane == 0) uf_unite(p.uf, (int32_t)c, nc, d);
        __syncwarp();
      }
    }
  }
}

// ------------------------------------------------------------------ k_ids
// Flatten every cell to its root (read-only walk, dbscan_cuda.cu:374-378) and
// rank the roots of non-noise components in cell order with a decoupled
// look-back exclusive scan (dbscan_cuda.cu:383-404, 698-701).
__global__ void __launch_bounds__(kScanThreads) k_ids(Plan p) {
  __shared__ uint32_t s_warp[kScanThreads / 32];
  __shared__ uint32_t s_tile;
  __shared__ unsigned long long s_excl;
  Desc* d = p.desc;
  const uint32_t C = d->num_cells;
  const int64_t tiles = ((int64_t)C + kScanTile - 1) / kScanTile;
  const uint32_t lane = lane_id(), warp = threadIdx.x >> 5;
  const int nwarps = blockDim.x >> 5;
  while (true) {
    if (threadIdx.x == 0) s_tile = atomicAdd(&d->ctr[kCtrIds], 1u);
    __syncthreads();
    const int64_t tile = s_tile;
    if (tile >= tiles) break;
    const int64_t c0 = tile * kScanTile + (int64_t)threadIdx.x * kScanItems;
    uint32_t flags = 0, cnt = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
      const int64_t c = c0 + k;
      if (c < C) {
        const int32_t r = uf_find_ro(p.uf, (int32_t)c, d);
        p.uf[c] = r;
        const bool f = r == (int32_t)c && p.cell_status[c] != 0;
        flags |= (uint32_t)f << k;
        cnt += f;
      }
    }
    uint32_t x = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(kFull, x, o);
      if (lane >= (uint32_t)o) x += y;
    }
    if (lane == 31) s_warp[warp] = x;
    __syncthreads();
    if (threadIdx.x == 0) {
      uint32_t run = 0;
      for (int wi = 0; wi < nwarps; ++wi) { const uint32_t t = s_warp[wi]; s_warp[wi] = run; run += t; }
      unsigned long long* my = p.ids_status + tile;
      unsigned long long excl = 0;
      if (tile == 0) st_relaxed(my, kFlagInc | run);
      else {
        st_relaxed(my, kFlagAgg | run);
        excl = lookback(p.ids_status, tile, 1, d);
        st_relaxed(my, kFlagInc | (excl + run));
      }
      s_excl = excl;
    }
    __syncthreads();
    uint32_t rnk = (uint32_t)s_excl + s_warp[warp] + x - cnt;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
      const int64_t c = c0 + k;
      if (c < C) {
        p.root_rank[c] = (int32_t)rnk;
        rnk += (flags >> k) & 1u;
      }
    }
    __syncthreads();
  }
}

// --------------------------------------------------------------- k_labels
// Per cell: cluster id of the cell (rank of its root among the cloud's
// roots), core labels, and for each non-core point the label of the nearest
// core point within eps, ties to the smaller input index (the (d2, perm[j])
// rule of dbscan_cuda.cu:447-467), written straight to input order.
constexpr int kQB = 4;  // queries per pass over the candidates

__device__ __forceinline__ int32_t cluster_of(const Plan& p, int32_t cell, int32_t seg_roots) {
  return p.cell_status[cell] == 0 ? -1 : p.root_rank[p.uf[cell]] - seg_roots;
}

__global__ void __launch_bounds__(kCellThreads) k_labels(Plan p) {
  __shared__ int32_t s_pre[kWarpsPerBlock][32];
  __shared__ int32_t s_off[kWarpsPerBlock][32];
  __shared__ int32_t s_lab[kWarpsPerBlock][32];
  const uint32_t lane = lane_id();
  const uint32_t w = threadIdx.x >> 5;
  Desc* d = p.desc;
  const uint32_t C = d->num_cells;
  while (true) {
    const uint32_t c = next_cell(&d->ctr[kCtrLabels]);
    if (c >= C) break;
    const int32_t seg = p.cell_seg[c];
    const int32_t seg_roots = p.root_rank[p.seg_info[seg].cell_begin];
    const uint8_t st = p.cell_status[c];
    const int32_t cid = st == 0 ? -1 : p.root_rank[p.uf[c]] - seg_roots;
    const int32_t st0 = p.cell_start[c], st1 = p.cell_start[c + 1];
    if (st == 2) {
      for (int32_t i = st0 + lane; i < st1; i += 32) p.labels[p.perm[i]] = cid;
      continue;
    }
    const float eps_sq = p.seg_param[seg].eps_sq;
    // Candidate cells: the 25 stencil cells (own cell included) with a core.
    int32_t nb = -1, sz = 0, cs0 = 0, lab = -1;
    float4 bb = make_float4(0.f, 0.f, 0.f, 0.f);
    if (lane < kNgh) {
      nb = p.ngh[(int64_t)c * kNgh + lane];
      if (nb >= 0 && p.cell_status[nb] != 0) {
        cs0 = p.cell_start[nb];
        sz = p.cell_start[nb + 1] - cs0;
        bb = p.bbox[nb];
        lab = cluster_of(p, nb, seg_roots);
      } else {
        nb = -1;
      }
    }
    s_lab[w][lane] = lab;
    for (int32_t ib = st0; ib < st1; ib += 32) {
      const int32_t i = ib + (int32_t)lane;
      const bool in = i < st1;
      const bool core = in && p.is_core[i];
      int32_t pi = 0;
      float2 q = make_float2(0.f, 0.f);
      if (in) { pi = (int32_t)p.perm[i]; q = p.xy[i]; }
      if (core) p.labels[pi] = cid;
      uint32_t qmask = __ballot_sync(kFull, in && !core);
      while (qmask) {
        // Up to kQB queries this pass.
        int ql[kQB];
        uint32_t mk[kQB];
        float qx[kQB], qy[kQB];
        uint32_t U = 0;
#pragma unroll
        for (int t = 0; t < kQB; ++t) {
          ql[t] = qmask ? __ffs(qmask) - 1 : -1;
          if (qmask) qmask &= qmask - 1;
          mk[t] = 0;
          qx[t] = 0.f; qy[t] = 0.f;
          if (ql[t] >= 0) {
            qx[t] = __shfl_sync(kFull, q.x, ql[t]);
            qy[t] = __shfl_sync(kFull, q.y, ql[t]);
            mk[t] = __ballot_sync(kFull, nb >= 0 && point_box_d2(qx[t], qy[t], bb) <= eps_sq);
            U |= mk[t];
          }
        }
        const int32_t szU = ((U >> lane) & 1u) ? sz : 0;
        const int32_t pre = warp_incl_scan(szU);
        const int32_t T = __shfl_sync(kFull, pre, 31);
        s_pre[w][lane] = pre;
        s_off[w][lane] = cs0 - (pre - szU);
        __syncwarp();
        unsigned long long best[kQB];
        int32_t blab[kQB];
#pragma unroll
        for (int t = 0; t < kQB; ++t) { best[t] = ~0ull; blab[t] = -1; }
        for (int32_t f0 = 0; f0 < T; f0 += 32) {
          const int32_t f = f0 + (int32_t)lane;
          if (f < T) {
            const int l = slice_of(s_pre[w], f);
            const int32_t j = f + s_off[w][l];
            if (p.is_core[j]) {
              const float2 pj = p.xy[j];
              const uint32_t pm = p.perm[j];
              const int32_t lj = s_lab[w][l];
#pragma unroll
              for (int t = 0; t < kQB; ++t) {
                if ((mk[t] >> l) & 1u) {
                  const float d2 = sq_dist(__fsub_rn(pj.x, qx[t]), __fsub_rn(pj.y, qy[t]));
                  if (d2 <= eps_sq) {
                    const unsigned long long key =
                        ((unsigned long long)__float_as_uint(d2) << 32) | pm;
                    if (key < best[t]) { best[t] = key; blab[t] = lj; }
                  }
                }
              }
            }
          }
        }
#pragma unroll
        for (int t = 0; t < kQB; ++t) {
          unsigned long long b = best[t];
          int32_t bl = blab[t];
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) {
            const unsigned long long ob = __shfl_xor_sync(kFull, b, o);
            const int32_t ol = __shfl_xor_sync(kFull, bl, o);
            if (ob < b) { b = ob; bl = ol; }
          }
          if (ql[t] >= 0 && (int)lane == ql[t]) p.labels[pi] = bl;
        }
        __syncwarp();
      }
    }
  }
}

// ------------------------------------------------------------- launchers
cudaError_t launch_core(const Plan& p, cudaStream_t s) {
  k_core<<<p.num_sms * 8, kCellThreads, 0, s>>>(p);
  return cudaGetLastError();
}

cudaError_t launch_union(const Plan& p, cudaStream_t s) {
  k_union<<<p.num_sms * 8, kCellThreads, 0, s>>>(p);
  return cudaGetLastError();
}

cudaError_t launch_ids(const Plan& p, cudaStream_t s) {
  k_ids<<<p.num_sms * 4, kScanThreads, 0, s>>>(p);
  return cudaGetLastError();
}

cudaError_t launch_labels(const Plan& p, cudaStream_t s) {
  k_labels<<<p.num_sms * 8, kCellThreads, 0, s>>>(p);
  return cudaGetLastError();
}

}  // namespace dbs
