// dbs_csort.cu -- counting sort of points by cell over a dense key space.
//
// Reference path replaced (ryanirl/dbscan-torch v0.2.0, csrc/cuda/dbscan_cuda.cu):
//   k_cell_keys :55-66, thrust::sort_by_key :582-586, k_gather_xy :71-79,
//   k_boundary_flags / inclusive_scan / k_extract_cell_start :84-120 and the
//   host read of num_cells :612-617.
//
// When the compacted key range is dense (every cloud within 6N + 4096 keys,
// or all clouds of a batch within that budget summed -- the rule that gives
// clouds a dense cell map), the sort needs no radix passes: a key *is* its
// bin. Two ordinary launches, then one cooperative kernel with phases
// separated by grid barriers:
//   0. clear the per-key counters (k_csort_clear)
//   1. count points per key (k_csort_count; atomics aggregated over lanes
//      with equal keys, so a 2M-point cell costs about one atomic per warp,
//      not per point). Outside the cooperative kernel, whose register
//      budget is set by the scan phases, the count runs at higher occupancy
//      (69 us instead of 105 us at 10M points).
//   2. per-block sums of counts and non-empty keys over contiguous key ranges
//   3. exclusive scan of the block sums (block 0)
//   4. rescan each range: the counter becomes the key's first output
//      position, the dense cell map gets each non-empty key's cell index, and
//      the cells get cell_start / cell_key / cell_seg (the run-length cells of
//      the reference, in the same ascending key order, without a pass over
//      sorted keys)
//   5. scatter every point's index to its key's next slot (perm); points of
//      hot keys (shared by >= kHotGroup lanes of one 32-point row) were
//      ranked by the count instead and go to the key's last slots without a
//      second fetch-add on the key
//   6. gather the sorted float2 coordinates point-parallel (coalesced writes)
// Points inside one cell land in arrival order rather than input order. No
// label depends on that order (core counts, cell-pair edges, boxes and the
// (d2, input index) border rule are all order-free), and cell indices are
// key ranks, identical to the reference's; only the debug entry point, which
// returns perm, forces the stable radix sort.
#include "dbs_internal.cuh"

namespace dbs {

constexpr int kCsThreads = 256;
constexpr uint32_t kFullMask = 0xffffffffu;

// Points per lane and iteration of the point loops: independent loads and
// atomics in flight per thread.
constexpr int kU = 4;

// Points per block of the cooperative kernel's grid (the grid grows with the
// cloud up to the resident blocks; a small cloud runs on few blocks, so its
// four grid barriers are cheap).
constexpr int64_t kCsPointsPerBlock = 2048;

// Warp aggregation of equal keys for the per-key atomics. __match_any_sync
// groups lanes with equal keys, but its cost grows with the number of
// distinct keys in the warp (about 7x a plain atomic's issue cost for 32
// distinct keys on B200). A warp first checks for duplicates between lanes
// l and l^16: warps of mostly distinct keys (the common case) skip the match
// and use one atomic per lane; warps with duplicates (a dense cell holding a
// large share of the points) group them so each key costs one atomic.
struct Agg {
  uint32_t group;   // lanes sharing this lane's atomic (bit set = member)
  uint32_t leader;  // lane that issues it
};

__device__ __forceinline__ Agg aggregate(uint32_t key, bool valid) {
  const uint32_t lane = lane_id();
  const uint32_t k = valid ? key : 0xffffffffu;
  // Every lane takes part in the shuffle (no short-circuit around a
  // warp-synchronous call).
  const uint32_t other = __shfl_xor_sync(kFullMask, k, 16);
  const bool dup = valid && k == other;
  Agg a;
  if (__ballot_sync(kFullMask, dup) == 0) {
    a.group = 1u << lane;
    a.leader = lane;
  } else {
    a.group = __match_any_sync(kFullMask, k);
    a.leader = __ffs(a.group) - 1;
  }
  return a;
}

// Hot-key table: open addressing with linear probing over a window of
// kHotProbes slots, insert-only, keyed by the dense key (< 2^31, so never
// kHotEmpty). The count kernel inserts: a key lands in the first slot of its
// window that is empty or holds it, so every inserter and every later reader
// agrees on the slot; later kernels only look keys up. A key whose window is
// full stays cold (correct, only slower). Probes read first and
// compare-and-swap only an empty slot, so once the table has filled (inputs
// in spatial order make most rows hot) a row costs a few L2 reads, not a
// queue of atomics on the table.
constexpr uint32_t kHotEmpty = 0xffffffffu;
constexpr int kHotProbes = 8;

__device__ __forceinline__ uint32_t hot_hash(uint32_t key) {
  return (key * 2654435761u) >> 26;  // multiplicative hash, top 6 bits
}

__device__ __forceinline__ int hot_insert(const Plan& p, uint32_t key) {
  uint32_t s = hot_hash(key);
  for (int probe = 0; probe < kHotProbes; ++probe, s = (s + 1) & (kHotSlots - 1)) {
    uint32_t k = __ldcg(&p.hot_key[s]);
    if (k == kHotEmpty) {
      k = atomicCAS(&p.hot_key[s], kHotEmpty, key);  // the slot's old value
      if (k == kHotEmpty) atomicAdd(&p.desc->hot_used, 1u);  // this lane took the slot
    }
    if (k == kHotEmpty || k == key) return (int)s;
  }
  return -1;
}

__device__ __forceinline__ int hot_find(const Plan& p, uint32_t key) {
  uint32_t s = hot_hash(key);
  for (int probe = 0; probe < kHotProbes; ++probe, s = (s + 1) & (kHotSlots - 1)) {
    const uint32_t k = p.hot_key[s];
    if (k == key) return (int)s;
    if (k == kHotEmpty) return -1;
  }
  return -1;
}

// Block-wide exclusive scan of two counters; returns the block totals.
__device__ __forceinline__ void block_scan2(uint32_t a, uint32_t b, uint32_t& xa, uint32_t& xb,
                                            uint32_t& ta, uint32_t& tb, uint32_t* s_a, uint32_t* s_b) {
  const uint32_t lane = lane_id(), warp = threadIdx.x >> 5;
  const int nw = blockDim.x >> 5;
  uint32_t ia = a, ib = b;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t ya = __shfl_up_sync(kFullMask, ia, o);
    const uint32_t yb = __shfl_up_sync(kFullMask, ib, o);
    if (lane >= (uint32_t)o) { ia += ya; ib += yb; }
  }
  if (lane == 31) { s_a[warp] = ia; s_b[warp] = ib; }
  __syncthreads();
  uint32_t pa = 0, pb = 0;
  ta = 0; tb = 0;
  for (int w = 0; w < nw; ++w) {
    if (w < (int)warp) { pa += s_a[w]; pb += s_b[w]; }
    ta += s_a[w]; tb += s_b[w];
  }
  xa = pa + ia - a;
  xb = pb + ib - b;
  __syncthreads();
}

// Exclusive scan of the per-key counts bins[0, W) of the dense key space
// (per-block range sums, a scan of the block sums by block 0, a rescan).
// Afterwards bins[b] is key b's first sorted position, and the cells exist:
// cell_map (key -> cell or -1), cell_start / cell_key / cell_seg, each
// cloud's cell_begin and num_cells. Cells are numbered in ascending key
// order, as the reference's run-length pass over sorted keys numbers them.
// Ends with a grid barrier.
__device__ __forceinline__ void scan_bins(const Plan& p, int64_t W, uint32_t* s_a, uint32_t* s_b) {
  Desc* d = p.desc;
  const int64_t n = p.n;
  uint32_t* bins = p.bin_count;
  constexpr int kI = 8;  // consecutive keys per thread in the rescan
  // Ranges of whole 8-key groups (16-byte aligned: bins and cell_map start
  // on 256-byte boundaries).
  const int64_t per = (((W + gridDim.x - 1) / gridDim.x) + kI - 1) & ~(int64_t)(kI - 1);
  const int64_t r0 = min(W, (int64_t)blockIdx.x * per), r1 = min(W, r0 + per);
  // Hot keys in this block's range: their count so far covers only the points
  // outside hot rows; add the hot rows' points (the block owns these keys, so
  // no other block reads or writes them here).
  if (threadIdx.x < kHotSlots) {
    const uint32_t key = p.hot_key[threadIdx.x];
    if (key != kHotEmpty && (int64_t)key >= r0 && (int64_t)key < r1) {
      const uint32_t cold = bins[key];
      p.hot_cold[threadIdx.x] = cold;
      bins[key] = cold + p.hot_cnt[threadIdx.x];
    }
  }
  __syncthreads();
  {
    uint32_t cs = 0, ne = 0;
    for (int64_t b = r0 + threadIdx.x; b < r1; b += blockDim.x) {
      const uint32_t c = bins[b];
      cs += c;
      ne += c != 0;
    }
    uint32_t xa, xb, ta, tb;
    block_scan2(cs, ne, xa, xb, ta, tb, s_a, s_b);
    if (threadIdx.x == 0) { p.blk_sum[blockIdx.x] = ta; p.blk_ne[blockIdx.x] = tb; }
  }
  grid_sync(&d->bar, d);

  // Exclusive scan of block sums (block 0; gridDim.x <= kMaxGrid).
  if (blockIdx.x == 0) {
    const int per_t = (gridDim.x + blockDim.x - 1) / blockDim.x;
    const int a0 = threadIdx.x * per_t, a1 = min((int)gridDim.x, a0 + per_t);
    uint32_t cs = 0, ne = 0;
    for (int k = a0; k < a1; ++k) { cs += p.blk_sum[k]; ne += p.blk_ne[k]; }
    uint32_t xa, xb, ta, tb;
    block_scan2(cs, ne, xa, xb, ta, tb, s_a, s_b);
    for (int k = a0; k < a1; ++k) {
      const uint32_t c = p.blk_sum[k], e = p.blk_ne[k];
      p.blk_sum[k] = xa;
      p.blk_ne[k] = xb;
      xa += c;
      xb += e;
    }
    if (threadIdx.x == 0) {
      d->num_cells = tb;
      p.cell_start[tb] = (int32_t)n;
    }
  }
  grid_sync(&d->bar, d);

  // Rescan: eight consecutive keys per thread (16-byte loads and stores),
  // one block scan per 8 * blockDim.x keys.
  {
    const bool one = p.nseg == 1;
    const uint64_t base0 = p.seg_info[0].base;
    uint32_t carry_cs = p.blk_sum[blockIdx.x], carry_ne = p.blk_ne[blockIdx.x];
    // Cloud of each key: one search for the thread's first key, then a walk
    // forward (a thread's keys only increase, so the walk covers each cloud
    // boundary once; a search per key cost a binary search over every cloud
    // for each of the 834M keys of a 4,096-cloud batch).
    int32_t sg = one ? 0 : seg_of_key(p, (uint64_t)min(r0 + (int64_t)threadIdx.x * kI, W > 0 ? W - 1 : 0));
    for (int64_t cb = r0; cb < r1; cb += (int64_t)blockDim.x * kI) {
      const int64_t b0 = cb + (int64_t)threadIdx.x * kI;
      const bool full = b0 + kI <= r1;
      uint32_t c[kI];
      if (full) {
        const uint4 lo = *reinterpret_cast<const uint4*>(bins + b0);
        const uint4 hi = *reinterpret_cast<const uint4*>(bins + b0 + 4);
        c[0] = lo.x; c[1] = lo.y; c[2] = lo.z; c[3] = lo.w;
        c[4] = hi.x; c[5] = hi.y; c[6] = hi.z; c[7] = hi.w;
      } else {
#pragma unroll
        for (int k = 0; k < kI; ++k) c[k] = b0 + k < r1 ? bins[b0 + k] : 0u;
      }
      uint32_t cs = 0, ne = 0;
#pragma unroll
      for (int k = 0; k < kI; ++k) { cs += c[k]; ne += c[k] != 0; }
      uint32_t xa, xb, ta, tb;
      block_scan2(cs, ne, xa, xb, ta, tb, s_a, s_b);
      uint32_t off = carry_cs + xa, cell = carry_ne + xb;
      uint32_t o[kI];
      int32_t m[kI];
#pragma unroll
      for (int k = 0; k < kI; ++k) {
        const int64_t b = b0 + k;
        o[k] = off;
        m[k] = c[k] ? (int32_t)cell : -1;
        if (b < r1) {
          if (!one)
            while (sg + 1 < p.nseg && p.seg_info[sg + 1].base <= (uint64_t)b) ++sg;
          if ((uint64_t)b == (one ? base0 : p.seg_info[sg].base)) p.seg_info[sg].cell_begin = (int32_t)cell;
          if (c[k]) {
            p.cell_start[cell] = (int32_t)off;
            p.cell_key[cell] = (uint64_t)b;
            p.cell_seg[cell] = sg;
          }
        }
        off += c[k];
        cell += c[k] != 0;
      }
      if (full) {
        *reinterpret_cast<uint4*>(bins + b0) = make_uint4(o[0], o[1], o[2], o[3]);
        *reinterpret_cast<uint4*>(bins + b0 + 4) = make_uint4(o[4], o[5], o[6], o[7]);
        *reinterpret_cast<int4*>(p.cell_map + b0) = make_int4(m[0], m[1], m[2], m[3]);
        *reinterpret_cast<int4*>(p.cell_map + b0 + 4) = make_int4(m[4], m[5], m[6], m[7]);
      } else {
#pragma unroll
        for (int k = 0; k < kI; ++k)
          if (b0 + k < r1) { bins[b0 + k] = o[k]; p.cell_map[b0 + k] = m[k]; }
      }
      carry_cs += ta;
      carry_ne += tb;
    }
  }
  // Hot points take the last slots of their key: after the cold points, which
  // the scatter places by fetch-add from the key's first slot.
  __syncthreads();
  if (threadIdx.x < kHotSlots) {
    const uint32_t key = p.hot_key[threadIdx.x];
    if (key != kHotEmpty && (int64_t)key >= r0 && (int64_t)key < r1)
      p.hot_base[threadIdx.x] = bins[key] + p.hot_cold[threadIdx.x];
  }
  grid_sync(&d->bar, d);
}

// Per-key counters cleared, then counted, by two ordinary launches before
// k_csort: outside the cooperative kernel they run at full occupancy (the
// counting loop needs far fewer registers than the scan phases).
__global__ void __launch_bounds__(kCsThreads) k_csort_clear(Plan p) {
  const Desc* d = p.desc;
  if (d->dense_sort != 1) return;
  const int64_t W = (int64_t)d->dense_total;
  const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t nthr = (int64_t)gridDim.x * blockDim.x;
  for (int64_t b = tid; b < W; b += nthr) p.bin_count[b] = 0;
  if (tid < kHotSlots) { p.hot_key[tid] = kHotEmpty; p.hot_cnt[tid] = 0; }
}

__global__ void __launch_bounds__(kCsThreads, 6) k_csort_count(Plan p) {
  const Desc* d = p.desc;
  if (d->dense_sort != 1) return;
  const int64_t n = p.n;
  uint32_t* bins = p.bin_count;
  const uint32_t lane = lane_id();
  const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t nthr = (int64_t)gridDim.x * blockDim.x;
  // Each warp takes kU consecutive 32-point rows per iteration;
  // peers = lanes with the same key, one atomic per peer group.
  const int64_t gwarp = tid >> 5, nwarps = nthr >> 5;
  {
    KeyCtx kc;
    kc.load(p, seg_of(p, min(gwarp * 32 * kU + lane, n > 0 ? n - 1 : 0)));
    for (int64_t base = gwarp * 32 * kU; base < n; base += nwarps * 32 * kU) {
      float2 v[kU];
#pragma unroll
      for (int k = 0; k < kU; ++k) {
        const int64_t i = base + k * 32 + lane;
        v[k] = i < n ? p.X[i] : make_float2(0.f, 0.f);
      }
#pragma unroll
      for (int k = 0; k < kU; ++k) {
        const int64_t i = base + k * 32 + lane;
        const bool valid = i < n;
        uint32_t key = 0xffffffffu;
        if (valid) {
          while (i >= kc.end) kc.load(p, kc.seg + 1);
          key = kc.key(v[k]);
        }
        const Agg a = aggregate(key, valid);
        const uint32_t g = (uint32_t)__popc(a.group);
        int slot = -1;
        uint32_t pos = 0;
        if (valid && lane == a.leader) {
          if (g >= kHotGroup) slot = hot_insert(p, key);
          if (slot >= 0) pos = atomicAdd(&p.hot_cnt[slot], g);
          else atomicAdd(&bins[key], g);
        }
        // Rows are the aligned 32-point groups [32m, 32m + 32) whatever the
        // grid, so the scatter sees the same groups and the same hot verdicts.
        if (__any_sync(kFullMask, slot >= 0)) {
          const int ls = __shfl_sync(kFullMask, slot, a.leader);
          const uint32_t b0 = __shfl_sync(kFullMask, pos, a.leader);
          if (valid && ls >= 0) p.vals[0][i] = b0 + __popc(a.group & lanemask_lt());
        }
      }
    }
  }
}

__global__ void __launch_bounds__(kCsThreads, 5) k_csort(Plan p) {
  __shared__ uint32_t s_a[kCsThreads / 32], s_b[kCsThreads / 32];
  Desc* d = p.desc;
  if (d->dense_sort != 1u) return;  // the radix sort ran
  const int64_t n = p.n;
  const int64_t W = (int64_t)d->dense_total;
  uint32_t* bins = p.bin_count;
  const uint32_t lane = lane_id();
  const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t nthr = (int64_t)gridDim.x * blockDim.x;

  const int64_t gwarp = tid >> 5, nwarps = nthr >> 5;
  mark_phase(d, 0);
  scan_bins(p, W, s_a, s_b);
  mark_phase(d, 3);

  // 5. scatter every point's input index to the slot its key's fetch-add
  //    returns (perm), or, in a hot row of a key in the hot table, to the
  //    key's hot base plus the rank the count kernel gave it
  {
    const uint32_t lt = lanemask_lt();
    KeyCtx kc;
    kc.load(p, seg_of(p, min(gwarp * 32 * kU + lane, n > 0 ? n - 1 : 0)));
    for (int64_t base = gwarp * 32 * kU; base < n; base += nwarps * 32 * kU) {
      float2 v[kU];
#pragma unroll
      for (int k = 0; k < kU; ++k) {
        const int64_t i = base + k * 32 + lane;
        v[k] = i < n ? p.X[i] : make_float2(0.f, 0.f);
      }
      uint32_t pos[kU];
      int hot[kU];
      Agg ag[kU];
#pragma unroll
      for (int k = 0; k < kU; ++k) {
        const int64_t i = base + k * 32 + lane;
        uint32_t key = 0xffffffffu;
        if (i < n) {
          while (i >= kc.end) kc.load(p, kc.seg + 1);
          key = kc.key(v[k]);
        }
        ag[k] = aggregate(key, i < n);
        pos[k] = 0;
        hot[k] = 0;
        if (i < n && lane == ag[k].leader) {
          const uint32_t g = (uint32_t)__popc(ag[k].group);
          const int slot = g >= kHotGroup ? hot_find(p, key) : -1;
          if (slot >= 0) {
            pos[k] = p.hot_base[slot];
            hot[k] = 1;
          } else {
            pos[k] = atomicAdd(&bins[key], g);
          }
        }
      }
#pragma unroll
      for (int k = 0; k < kU; ++k) {
        const int64_t i = base + k * 32 + lane;
        const int h = __shfl_sync(kFullMask, hot[k], ag[k].leader);
        uint32_t at = __shfl_sync(kFullMask, pos[k], ag[k].leader);
        if (i < n) {
          at += h ? p.vals[0][i] : (uint32_t)__popc(ag[k].group & lt);
          if ((int64_t)at < n) p.perm[at] = (uint32_t)i;
          else set_error(d, kErrCapacity);
        }
      }
    }
  }
  grid_sync(&d->bar, d);
  mark_phase(d, 4);

  // 6. gather the sorted coordinates (the reference's k_gather_xy):
  //    coalesced perm reads and xy writes, independent random reads of X.
  //    (Writing the coordinates in the scatter instead costs more: random
  //    8-byte writes leave partial sectors.)
  for (int64_t i0 = tid; i0 < n; i0 += nthr * kU) {
    uint32_t src[kU];
#pragma unroll
    for (int k = 0; k < kU; ++k) {
      const int64_t i = i0 + k * nthr;
      src[k] = i < n ? p.perm[i] : 0u;
    }
#pragma unroll
    for (int k = 0; k < kU; ++k) {
      const int64_t i = i0 + k * nthr;
      if (i < n) p.xy[i] = p.X[src[k]];
    }
  }
  __syncthreads();
  mark_phase(d, 5);
}

cudaError_t launch_csort(const Plan& p, cudaStream_t s) {
  static PerDeviceBlocks cache;
  int blocks_per_sm = 0;
  cudaError_t e = cache.get(
      [](int* b) { return cudaOccupancyMaxActiveBlocksPerMultiprocessor(b, k_csort, kCsThreads, 0); },
      &blocks_per_sm);
  if (e != cudaSuccess) return e;
  k_csort_clear<<<p.num_sms * 4, kCsThreads, 0, s>>>(p);
  k_csort_count<<<p.num_sms * p.bps[kTuneCount], kCsThreads, 0, s>>>(p);
  const int grid = coop_grid((p.n + kCsPointsPerBlock - 1) / kCsPointsPerBlock, p.num_sms,
                             p.num_sms * blocks_per_sm);
  Plan q = p;
  void* args[] = {&q};
  return cudaLaunchCooperativeKernel((const void*)k_csort, dim3(grid), dim3(kCsThreads), args, 0, s);
}

}  // namespace dbs
