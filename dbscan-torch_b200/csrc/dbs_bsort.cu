// dbs_bsort.cu -- bucketed counting sort of points by cell over a dense key space.
//
// Reference path replaced (ryanirl/dbscan-torch v0.2.0, csrc/cuda/dbscan_cuda.cu):
//   k_cell_keys :55-66, thrust::sort_by_key :582-586, k_gather_xy :71-79,
//   k_boundary_flags / inclusive_scan / k_extract_cell_start :84-120 and the
//   host read of num_cells :612-617.
//
// The global counting sort (dbs_csort.cu) costs four random global
// transactions per point: a count atomic, a fetch-add, a 4-byte scatter into
// perm and an 8-byte gather of the coordinates. On a shuffled cloud each one
// lands on a different sector, so that sort runs at the rate of random L2
// transactions, not of HBM. This sort moves every point twice in streams
// instead:
//
//   k_bkt_part (cooperative, one contiguous chunk of points per block)
//     1. per-chunk histogram of buckets (2^bkt_shift consecutive keys each)
//        in shared memory, written as a bucket-major (bucket, chunk) matrix
//     2. exclusive scan of each bucket's row over the chunks
//     3. block 0: exclusive scan of the bucket totals (bucket starts); the
//        largest bucket decides the form: at most kBktCap points -> this
//        sort, else the global counting sort runs instead (few huge cells)
//     4. partition: each block re-reads its chunk tile by tile, ranks the
//        tile's points by bucket in shared memory, stages them in bucket
//        order and writes each bucket's run of records (input index, x, y;
//        and the key for multi-cloud runs) at the chunk's next slot of that
//        bucket. Consecutive threads write consecutive records of a run.
//   k_bkt_local (one block per bucket, buckets taken in order)
//     5. counts of the bucket's keys in shared memory (a stream over the
//        bucket's records, which stay in L2 for step 7)
//     6. exclusive scan of the counts; the bucket's first cell index comes
//        from a decoupled look-back over the buckets' non-empty key counts;
//        the bucket writes its cells (cell_start, cell_key, cell_seg, each
//        cloud's cell_begin) and its slice of the dense cell map
//     7. places each record at its key's next slot inside the bucket's
//        range: perm and the sorted coordinates, random only within a range
//        of a few tens of kilobytes, whose sectors fill in L2
//
// As in the global counting sort, points inside a cell land in arrival
// order, cells are numbered in ascending key order (the reference's
// run-length order) and no label depends on the order inside a cell.
// Eligible: dense key spaces (the counting sort's rule) of runs with at least
// kBktMinPoints points whose key range splits into at most kBktMaxBuckets
// buckets of at most kBktMaxKeys keys (k_seg_finalize decides).
#include "dbs_internal.cuh"

namespace dbs {

namespace {

constexpr uint32_t kFull = 0xffffffffu;
constexpr int kBktWarps = kBktThreads / 32;
constexpr int kPartItems = kBktTile / kBktThreads;  // points per thread per tile
constexpr int kLocalItems = 8;                      // records per thread per step of the local pass

// Dynamic shared memory of k_bkt_part.
struct PartSmem {
  uint32_t cnt[kBktMaxBuckets + 1];    // tile counts per bucket -> tile offsets
  uint32_t carry[kBktMaxBuckets];      // chunk's next record of each bucket
  uint32_t warp_tot[kBktWarps];
  uint32_t s_idx[kBktTile];            // staged records, bucket order
  uint32_t s_key[kBktTile];
  float2 s_xy[kBktTile];
};

__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t v) {
  const uint32_t lane = lane_id();
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(kFull, v, o);
    if (lane >= (uint32_t)o) v += y;
  }
  return v;
}

// In-place exclusive scan of a[0, m) in shared memory by the whole block;
// a[m] receives the total, which is also returned. Warp w owns a contiguous
// segment and walks it in 32-entry chunks (lane-contiguous, conflict-free).
__device__ uint32_t block_exscan(uint32_t* a, int m, uint32_t* warp_tot) {
  const int nw = blockDim.x >> 5;
  const int warp = threadIdx.x >> 5, lane = (int)lane_id();
  const int seg = (((m + nw - 1) / nw) + 31) & ~31;
  const int lo = min(m, warp * seg), hi = min(m, lo + seg);
  uint32_t t = 0;
  for (int j = lo + lane; j < hi; j += 32) t += a[j];
  t = __reduce_add_sync(kFull, t);
  if (lane == 0) warp_tot[warp] = t;
  __syncthreads();
  uint32_t pre = 0, tot = 0;
  for (int w = 0; w < nw; ++w) {
    const uint32_t v = warp_tot[w];
    if (w < warp) pre += v;
    tot += v;
  }
  uint32_t run = pre;
  for (int base = lo; base < hi; base += 32) {
    const int j = base + lane;
    const uint32_t v = j < hi ? a[j] : 0u;
    const uint32_t x = warp_incl_scan(v);
    if (j < hi) a[j] = run + x - v;
    run += __shfl_sync(kFull, x, 31);
  }
  if (threadIdx.x == 0) a[m] = tot;
  __syncthreads();
  return tot;
}

}  // namespace

// ------------------------------------------------------------- k_bkt_part
__global__ void __launch_bounds__(kBktThreads, 2) k_bkt_part(Plan p) {
  extern __shared__ __align__(16) unsigned char bkt_smem[];
  PartSmem& sm = *reinterpret_cast<PartSmem*>(bkt_smem);
  Desc* d = p.desc;
  if (!d->bkt_ok) return;  // uniform over the grid: no barrier is reached
  const int64_t n = p.n;
  const uint32_t shift = d->bkt_shift;
  const int NB = (int)d->bkt_nb;
  const int G = (int)gridDim.x;
  const int c = (int)blockIdx.x;
  const int64_t per = (n + G - 1) / G;
  const int64_t c0 = min(n, (int64_t)c * per), c1 = min(n, c0 + per);
  const bool multi = p.nseg > 1;
  uint32_t* const rec_idx = p.vals[0];
  float2* const rec_xy = reinterpret_cast<float2*>(p.keys[0]);
  uint32_t* const rec_key = reinterpret_cast<uint32_t*>(p.keys[1]);
  mark_phase(d, 0);

  // 1. histogram of this chunk's buckets (kPartItems independent loads in
  //    flight per thread, as in the partition)
  for (int b = threadIdx.x; b < NB; b += blockDim.x) sm.cnt[b] = 0;
  __syncthreads();
  if (c0 < c1) {
    KeyCtx kc;
    kc.load(p, seg_of(p, c0 + min((int64_t)threadIdx.x, c1 - c0 - 1)));
    for (int64_t tile = c0; tile < c1; tile += kBktTile) {
      float2 v[kPartItems];
#pragma unroll
      for (int k = 0; k < kPartItems; ++k) {
        const int64_t i = tile + k * kBktThreads + threadIdx.x;
        v[k] = i < c1 ? p.X[i] : make_float2(0.f, 0.f);
      }
#pragma unroll
      for (int k = 0; k < kPartItems; ++k) {
        const int64_t i = tile + k * kBktThreads + threadIdx.x;
        if (i < c1) {
          while (i >= kc.end) kc.load(p, kc.seg + 1);
          atomicAdd(&sm.cnt[kc.key(v[k]) >> shift], 1u);
        }
      }
    }
  }
  __syncthreads();
  for (int b = threadIdx.x; b < NB; b += blockDim.x) p.bkt_mat[(int64_t)b * G + c] = sm.cnt[b];
  grid_sync(&d->bar, d);
  mark_phase(d, 1);

  // 2. exclusive scan of each bucket's row over the chunks (a warp per row)
  {
    const int gw = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int nwarps = (int)((gridDim.x * blockDim.x) >> 5);
    for (int b = gw; b < NB; b += nwarps) {
      uint32_t* row = p.bkt_mat + (int64_t)b * G;
      uint32_t run = 0;
      for (int base = 0; base < G; base += 32) {
        const int j = base + (int)lane_id();
        const uint32_t v = j < G ? row[j] : 0u;
        const uint32_t x = warp_incl_scan(v);
        if (j < G) row[j] = run + x - v;
        run += __shfl_sync(kFull, x, 31);
      }
      if (lane_id() == 0) p.bkt_tot[b] = run;
    }
  }
  grid_sync(&d->bar, d);

  // 3. bucket starts and the form (block 0)
  if (blockIdx.x == 0) {
    uint32_t mx = 0;
    for (int b = threadIdx.x; b < NB; b += blockDim.x) {
      const uint32_t v = p.bkt_tot[b];
      sm.cnt[b] = v;
      mx = max(mx, v);
      p.bkt_status[b] = 0ull;
    }
    mx = __reduce_max_sync(kFull, mx);
    if (lane_id() == 0) sm.warp_tot[threadIdx.x >> 5] = mx;
    __syncthreads();
    if (threadIdx.x == 0) {
      uint32_t m = 0;
      for (int w = 0; w < kBktWarps; ++w) m = max(m, sm.warp_tot[w]);
      d->bkt_max = m;
      d->dense_sort = m <= kBktCap ? 2u : 1u;
    }
    __syncthreads();
    block_exscan(sm.cnt, NB, sm.warp_tot);
    for (int b = threadIdx.x; b <= NB; b += blockDim.x) p.bkt_start[b] = sm.cnt[b];
  }
  grid_sync(&d->bar, d);
  mark_phase(d, 2);
  if (*reinterpret_cast<volatile uint32_t*>(&d->dense_sort) != 2u) return;

  // 4. partition: records of this chunk into their buckets' runs
  for (int b = threadIdx.x; b < NB; b += blockDim.x)
    sm.carry[b] = p.bkt_start[b] + p.bkt_mat[(int64_t)b * G + c];
  KeyCtx kc;
  if (c0 < c1) kc.load(p, seg_of(p, c0 + min((int64_t)threadIdx.x, c1 - c0 - 1)));
  for (int64_t tile = c0; tile < c1; tile += kBktTile) {
    const int valid = (int)min((int64_t)kBktTile, c1 - tile);
    for (int b = threadIdx.x; b < NB; b += blockDim.x) sm.cnt[b] = 0;
    __syncthreads();
    uint32_t key[kPartItems], rank[kPartItems];
    float2 v[kPartItems];
#pragma unroll
    for (int k = 0; k < kPartItems; ++k) {
      const int64_t i = tile + k * kBktThreads + threadIdx.x;
      v[k] = i < c1 ? p.X[i] : make_float2(0.f, 0.f);
    }
#pragma unroll
    for (int k = 0; k < kPartItems; ++k) {
      const int64_t i = tile + k * kBktThreads + threadIdx.x;
      if (i < c1) {
        while (i >= kc.end) kc.load(p, kc.seg + 1);
        key[k] = kc.key(v[k]);
        rank[k] = atomicAdd(&sm.cnt[key[k] >> shift], 1u);
      }
    }
    __syncthreads();
    block_exscan(sm.cnt, NB, sm.warp_tot);
#pragma unroll
    for (int k = 0; k < kPartItems; ++k) {
      const int64_t i = tile + k * kBktThreads + threadIdx.x;
      if (i < c1) {
        const uint32_t lp = sm.cnt[key[k] >> shift] + rank[k];
        sm.s_idx[lp] = (uint32_t)i;
        sm.s_key[lp] = key[k];
        sm.s_xy[lp] = v[k];
      }
    }
    __syncthreads();
    for (int lp = threadIdx.x; lp < valid; lp += blockDim.x) {
      const uint32_t kk = sm.s_key[lp];
      const uint32_t b = kk >> shift;
      const uint32_t g = sm.carry[b] + (uint32_t)lp - sm.cnt[b];
      rec_idx[g] = sm.s_idx[lp];
      rec_xy[g] = sm.s_xy[lp];
      if (multi) rec_key[g] = kk;
    }
    __syncthreads();
    for (int b = threadIdx.x; b < NB; b += blockDim.x) sm.carry[b] += sm.cnt[b + 1] - sm.cnt[b];
    __syncthreads();
  }
  mark_phase(d, 3);
}

// ------------------------------------------------------------ k_bkt_local
__global__ void __launch_bounds__(kBktThreads) k_bkt_local(Plan p) {
  __shared__ uint32_t s_cnt[kBktMaxKeys + 1];
  __shared__ uint32_t s_wpts[kBktWarps], s_wne[kBktWarps];
  __shared__ uint32_t s_ticket;
  __shared__ unsigned long long s_base;
  Desc* d = p.desc;
  if (d->dense_sort != 2u) return;
  const int64_t n = p.n;
  const uint32_t NB = d->bkt_nb, shift = d->bkt_shift;
  const int64_t W = (int64_t)d->dense_total;
  const bool one = p.nseg == 1;
  const uint32_t* const rec_idx = p.vals[0];
  const float2* const rec_xy = reinterpret_cast<const float2*>(p.keys[0]);
  const uint32_t* const rec_key = reinterpret_cast<const uint32_t*>(p.keys[1]);
  const int warp = threadIdx.x >> 5, lane = (int)lane_id();
  KeyCtx kc0;
  if (one) kc0.load(p, 0);
  const uint64_t base0 = p.seg_info[0].base;
  while (true) {
    if (threadIdx.x == 0) s_ticket = atomicAdd(&d->ctr[kCtrBkt], 1u);
    __syncthreads();
    const uint32_t b = s_ticket;
    if (b >= NB) break;
    const int64_t kb0 = (int64_t)b << shift;
    const int kn = (int)min((int64_t)1 << shift, W - kb0);
    const uint32_t rs = p.bkt_start[b], re = p.bkt_start[b + 1];
    for (int k = threadIdx.x; k < kn; k += blockDim.x) s_cnt[k] = 0;
    __syncthreads();

    // 5. key counts (kLocalItems independent loads in flight per thread)
    for (uint32_t r0 = rs; r0 < re; r0 += kLocalItems * kBktThreads) {
      uint32_t key[kLocalItems];
#pragma unroll
      for (int k = 0; k < kLocalItems; ++k) {
        const uint32_t r = r0 + k * kBktThreads + threadIdx.x;
        if (r < re) key[k] = one ? kc0.key(rec_xy[r]) : rec_key[r];
      }
#pragma unroll
      for (int k = 0; k < kLocalItems; ++k) {
        const uint32_t r = r0 + k * kBktThreads + threadIdx.x;
        if (r < re) atomicAdd(&s_cnt[key[k] - (uint32_t)kb0], 1u);
      }
    }
    __syncthreads();

    // 6. scan of points and non-empty keys; the bucket's first cell
    const int seg = (((kn + kBktWarps - 1) / kBktWarps) + 31) & ~31;
    const int lo = min(kn, warp * seg), hi = min(kn, lo + seg);
    uint32_t tp = 0, te = 0;
    for (int j = lo + lane; j < hi; j += 32) {
      const uint32_t v = s_cnt[j];
      tp += v;
      te += v != 0u;
    }
    tp = __reduce_add_sync(kFull, tp);
    te = __reduce_add_sync(kFull, te);
    if (lane == 0) { s_wpts[warp] = tp; s_wne[warp] = te; }
    __syncthreads();
    if (warp == 0) {
      uint32_t ne_tot = 0;
      for (int w = 0; w < kBktWarps; ++w) ne_tot += s_wne[w];
      unsigned long long* my = p.bkt_status + b;
      unsigned long long excl = 0;
      if (b == 0) {
        if (lane == 0) st_relaxed(my, kFlagInc | ne_tot);
      } else {
        if (lane == 0) st_relaxed(my, kFlagAgg | ne_tot);
        excl = lookback_warp(p.bkt_status, b, 1, d);
        if (lane == 0) st_relaxed(my, kFlagInc | (excl + ne_tot));
      }
      if (lane == 0) {
        s_base = excl;
        if (b == NB - 1) {
          uint32_t total = (uint32_t)(excl + ne_tot);
          if ((int64_t)total > n) total = (uint32_t)n;  // only after a failed look-back
          d->num_cells = total;
          p.cell_start[total] = (int32_t)n;
        }
      }
    }
    __syncthreads();
    {
      uint32_t pre_p = 0, pre_e = 0;
      for (int w = 0; w < warp; ++w) { pre_p += s_wpts[w]; pre_e += s_wne[w]; }
      uint32_t cell = (uint32_t)s_base + pre_e;  // next cell index in this warp's segment
      uint32_t off = pre_p;                       // next record offset inside the bucket
      for (int base = lo; base < hi; base += 32) {
        const int j = base + lane;
        const uint32_t v = j < hi ? s_cnt[j] : 0u;
        const uint32_t ne = v != 0u ? 1u : 0u;
        const uint32_t xp = warp_incl_scan(v);
        const uint32_t xe = warp_incl_scan(ne);
        const uint32_t my_off = off + xp - v;
        const uint32_t my_cell = cell + xe - ne;
        if (j < hi) {
          const int64_t key = kb0 + j;
          s_cnt[j] = my_off;
          p.cell_map[key] = v ? (int32_t)my_cell : -1;
          int32_t sg = 0;
          if (!one) {
            sg = seg_of_key(p, (uint64_t)key);
            if ((uint64_t)key == p.seg_info[sg].base) p.seg_info[sg].cell_begin = (int32_t)my_cell;
          } else if ((uint64_t)key == base0) {
            p.seg_info[0].cell_begin = (int32_t)my_cell;
          }
          if (v && (int64_t)my_cell < n) {
            p.cell_start[my_cell] = (int32_t)(rs + my_off);
            p.cell_key[my_cell] = (uint64_t)key;
            p.cell_seg[my_cell] = sg;
          }
        }
        off += __shfl_sync(kFull, xp, 31);
        cell += __shfl_sync(kFull, xe, 31);
      }
    }
    __syncthreads();

    // 7. place the records (loads batched as in step 5)
    for (uint32_t r0 = rs; r0 < re; r0 += kLocalItems * kBktThreads) {
      float2 v[kLocalItems];
      uint32_t key[kLocalItems], idx[kLocalItems];
#pragma unroll
      for (int k = 0; k < kLocalItems; ++k) {
        const uint32_t r = r0 + k * kBktThreads + threadIdx.x;
        if (r < re) {
          v[k] = rec_xy[r];
          idx[k] = rec_idx[r];
          if (!one) key[k] = rec_key[r];
        }
      }
#pragma unroll
      for (int k = 0; k < kLocalItems; ++k) {
        const uint32_t r = r0 + k * kBktThreads + threadIdx.x;
        if (r < re) {
          const uint32_t kk = one ? kc0.key(v[k]) : key[k];
          const uint32_t at = rs + atomicAdd(&s_cnt[kk - (uint32_t)kb0], 1u);
          if (at < re) {
            p.perm[at] = idx[k];
            p.xy[at] = v[k];
          } else {
            set_error(d, kErrCapacity);
          }
        }
      }
    }
    __syncthreads();
  }
}

// ------------------------------------------------------------- launchers
constexpr size_t kPartSmemBytes = sizeof(PartSmem);

// Cooperative partition (grid = resident blocks, at most kBktMaxChunks)
// and the local pass; both return at once unless the bucketed sort runs.
cudaError_t launch_bsort(const Plan& p, cudaStream_t s) {
  static PerDeviceBlocks cache;
  int blocks_per_sm = 0;
  cudaError_t e = cache.get(
      [](int* b) {
        cudaError_t r = cudaFuncSetAttribute(k_bkt_part, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)kPartSmemBytes);
        if (r != cudaSuccess) return r;
        return cudaOccupancyMaxActiveBlocksPerMultiprocessor(b, k_bkt_part, kBktThreads, kPartSmemBytes);
      },
      &blocks_per_sm);
  if (e != cudaSuccess) return e;
  int grid = p.num_sms * blocks_per_sm;
  if (grid > kBktMaxChunks) grid = kBktMaxChunks;
  Plan q = p;
  void* args[] = {&q};
  e = cudaLaunchCooperativeKernel((const void*)k_bkt_part, dim3(grid), dim3(kBktThreads), args,
                                  kPartSmemBytes, s);
  if (e != cudaSuccess) return e;
  k_bkt_local<<<p.num_sms * 8, kBktThreads, 0, s>>>(p);
  return cudaGetLastError();
}

}  // namespace dbs
