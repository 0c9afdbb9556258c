// dbs_sort.cu -- per-cloud key layout and the LSD radix sort.
//
// Reference path replaced (ryanirl/dbscan-torch v0.2.0, csrc/cuda/dbscan_cuda.cu):
//   k_cell_keys :55-66, thrust::sort_by_key :582-586, k_gather_xy :71-79.
//
// Keys. The reference sorts u64 keys (u32)kx << 32 | (u32)ky. Here each cloud
// first reduces the bounds of its cell coordinates, split into the
// non-negative and the negative class per axis; the compacted coordinate
// (non-negative class first, then the negative class, each ascending) is a
// strictly increasing function of the u32 coordinate, so
//   key = base[cloud] + gx * wy + gy
// sorts exactly like the reference key while needing only
// ceil(log2(sum of ranges)) bits: 22 bits (three 8-bit passes) for a
// 10M-point constant-density cloud instead of eight passes. Keys are stored
// as u32 when they fit, else u64 (decided on the device).
//
// Sort (clouds whose key range is sparse, and the debug entry point; dense
// key spaces take the counting sort of dbs_csort.cu): k_keys writes the keys
// and the first digit's counts per chunk; k_radix, one cooperative kernel,
// runs the LSD passes with 8-bit digits -- per-digit scan of the chunk counts,
// then each chunk ranks each 4096-key tile in shared memory (ballot-based,
// stable) and scatters through a shared-memory staging buffer so each digit
// run is written contiguously. The last pass writes perm and gathers the
// float2 coordinates (the reference's k_gather_xy) in the same scatter.
#include "dbs_internal.cuh"

namespace dbs {

// ----------------------------------------------------------------- k_init
__global__ void k_init(Plan p) {
  const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  Desc* d = p.desc;
  if (tid == 0) {
    d->status = 0;
    d->key64 = 0;
    d->nbits = 0;
    d->npasses = 1;
    d->num_cells = 0;
    d->dense_total = 0;
    d->big_packed = 0;
  }
  for (int64_t i = tid; i < 2 * kRadix; i += stride) (&d->digit_total[0][0])[i] = 0;
  if (tid == 0) {
    d->bar.count = 0; d->bar.gen = 0; d->dense_sort = 0;
    d->q_count = 0; d->b_count = 0; d->p_count = 0; d->d_count = 0; d->hot_used = 0;
    d->ring_pairs[0] = d->ring_pairs[1] = 0; d->ring_warp[0] = d->ring_warp[1] = 0;
  }
  for (int64_t i = tid; i < p.scan_tiles; i += stride) p.rle_status[i] = 0;
  for (int64_t i = tid; i < p.ids_tiles; i += stride) p.ids_status[i] = 0;
  if (p.single && tid == 0) {
    p.seg_off[0] = 0;
    p.seg_off[1] = p.n;
    p.seg_param[0] = p.single_param;
  }
  for (int64_t i = tid; i < kNumCtr; i += stride) d->ctr[i] = 0;
  for (int64_t s = tid; s < p.nseg; s += stride) {
    SegInfo& g = p.seg_info[s];
    g.bx[0] = INT32_MAX; g.bx[1] = -1; g.bx[2] = 0; g.bx[3] = INT32_MIN;
    g.by[0] = INT32_MAX; g.by[1] = -1; g.by[2] = 0; g.by[3] = INT32_MIN;
    g.cell_begin = 0;
  }
}

// --------------------------------------------------------------- k_bounds
// Per-cloud class bounds. Each thread folds a run of points of one cloud and
// flushes with atomics when the cloud changes.
struct AxisAcc {
  int32_t lo_pos, hi_pos, lo_neg, hi_neg;
  __device__ void reset() { lo_pos = INT32_MAX; hi_pos = -1; lo_neg = 0; hi_neg = INT32_MIN; }
  __device__ void add(int32_t k) {
    if (k >= 0) { lo_pos = min(lo_pos, k); hi_pos = max(hi_pos, k); }
    else { lo_neg = min(lo_neg, k); hi_neg = max(hi_neg, k); }
  }
  __device__ void flush(int32_t* b) {
    if (hi_pos >= 0) { atomicMin(&b[0], lo_pos); atomicMax(&b[1], hi_pos); }
    if (lo_neg < 0) { atomicMin(&b[2], lo_neg); atomicMax(&b[3], hi_neg); }
  }
};

__device__ __forceinline__ void warp_fold(AxisAcc& a) {
  const uint32_t full = 0xffffffffu;
  a.lo_pos = __reduce_min_sync(full, a.lo_pos);
  a.hi_pos = __reduce_max_sync(full, a.hi_pos);
  a.lo_neg = __reduce_min_sync(full, a.lo_neg);
  a.hi_neg = __reduce_max_sync(full, a.hi_neg);
}

__global__ void __launch_bounds__(256) k_bounds(Plan p) {
  const int64_t n = p.n;
  // Each block owns a contiguous chunk; within it, lanes read consecutive
  // points (coalesced float2 loads).
  const int64_t per_block = (n + gridDim.x - 1) / gridDim.x;
  const int64_t b0 = (int64_t)blockIdx.x * per_block;
  const int64_t b1 = min(n, b0 + per_block);
  if (b0 >= b1) return;
  int32_t seg = seg_of(p, b0);
  int64_t seg_end = p.seg_off[seg + 1];
  float inv_r = p.seg_param[seg].inv_r;
  AxisAcc ax, ay;
  ax.reset(); ay.reset();
  if (b1 <= seg_end) {
    // The whole chunk lies in one cloud (every chunk of a plain call): four
    // independent loads per thread in flight, then one flush per block.
    __shared__ int32_t s_b[8];
    if (threadIdx.x < 8) {  // lo_pos, hi_pos, lo_neg, hi_neg of x, then of y (AxisAcc::reset)
      const int32_t r = threadIdx.x & 3;
      s_b[threadIdx.x] = r == 0 ? INT32_MAX : r == 1 ? -1 : r == 2 ? 0 : INT32_MIN;
    }
    constexpr int kB = 4;
    int64_t base = b0;
    for (; base + kB * (int64_t)blockDim.x <= b1; base += kB * (int64_t)blockDim.x) {
      float2 v[kB];
#pragma unroll
      for (int k = 0; k < kB; ++k) v[k] = p.X[base + k * (int64_t)blockDim.x + threadIdx.x];
#pragma unroll
      for (int k = 0; k < kB; ++k) {
        ax.add(cell_coord(v[k].x, inv_r));
        ay.add(cell_coord(v[k].y, inv_r));
      }
    }
    for (int64_t i = base + threadIdx.x; i < b1; i += blockDim.x) {
      const float2 v = p.X[i];
      ax.add(cell_coord(v.x, inv_r));
      ay.add(cell_coord(v.y, inv_r));
    }
    warp_fold(ax); warp_fold(ay);
    __syncthreads();
    if (lane_id() == 0) {
      atomicMin(&s_b[0], ax.lo_pos); atomicMax(&s_b[1], ax.hi_pos);
      atomicMin(&s_b[2], ax.lo_neg); atomicMax(&s_b[3], ax.hi_neg);
      atomicMin(&s_b[4], ay.lo_pos); atomicMax(&s_b[5], ay.hi_pos);
      atomicMin(&s_b[6], ay.lo_neg); atomicMax(&s_b[7], ay.hi_neg);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      AxisAcc bx{s_b[0], s_b[1], s_b[2], s_b[3]}, by{s_b[4], s_b[5], s_b[6], s_b[7]};
      bx.flush(p.seg_info[seg].bx);
      by.flush(p.seg_info[seg].by);
    }
    return;
  }
  for (int64_t base = b0; base < b1; base += blockDim.x) {
    const int64_t i = base + threadIdx.x;
    // The cloud of the whole block-row: when the row is inside one cloud
    // (the common case) the warp folds its partial bounds before flushing.
    while (base >= seg_end) {
      // block-uniform advance to the cloud containing `base`
      ++seg;
      seg_end = p.seg_off[seg + 1];
      inv_r = p.seg_param[seg].inv_r;
    }
    const bool row_in_seg = (min(base + (int64_t)blockDim.x, b1) <= seg_end);
    if (row_in_seg) {
      if (i < b1) {
        float2 v = p.X[i];
        ax.add(cell_coord(v.x, inv_r));
        ay.add(cell_coord(v.y, inv_r));
      }
    } else {
      // Row straddles clouds: fold the running accumulators first, then
      // handle each point with its own cloud's atomics.
      warp_fold(ax); warp_fold(ay);
      if (lane_id() == 0) { ax.flush(p.seg_info[seg].bx); ay.flush(p.seg_info[seg].by); }
      ax.reset(); ay.reset();
      if (i < b1) {
        const int32_t s = seg_of(p, i);
        const float ir = p.seg_param[s].inv_r;
        float2 v = p.X[i];
        AxisAcc tx, ty;
        tx.reset(); ty.reset();
        tx.add(cell_coord(v.x, ir));
        ty.add(cell_coord(v.y, ir));
        tx.flush(p.seg_info[s].bx);
        ty.flush(p.seg_info[s].by);
      }
      // Continue with the cloud of the last point of this row.
      const int64_t last = min(base + (int64_t)blockDim.x, b1) - 1;
      while (last >= seg_end) {
        ++seg;
        seg_end = p.seg_off[seg + 1];
        inv_r = p.seg_param[seg].inv_r;
      }
    }
    // Flush when the next row starts in another cloud.
    const int64_t next = base + blockDim.x;
    if (next < b1 && next >= seg_end) {
      warp_fold(ax); warp_fold(ay);
      if (lane_id() == 0) { ax.flush(p.seg_info[seg].bx); ay.flush(p.seg_info[seg].by); }
      ax.reset(); ay.reset();
    }
  }
  warp_fold(ax); warp_fold(ay);
  if (lane_id() == 0) { ax.flush(p.seg_info[seg].bx); ay.flush(p.seg_info[seg].by); }
}

// --------------------------------------------------------- k_seg_finalize
// One block: per-cloud class widths, key bases (exclusive scan of the
// per-cloud ranges), dense-map bases, and the global key width.
__global__ void __launch_bounds__(1024) k_seg_finalize(Plan p) {
  __shared__ unsigned long long s_range[1024];
  __shared__ unsigned long long s_dense[1024];
  __shared__ unsigned long long s_carry_range, s_carry_dense;
  __shared__ int s_overflow, s_sparse;
  if (threadIdx.x == 0) { s_carry_range = 0; s_carry_dense = 0; s_overflow = 0; s_sparse = 0; }
  __syncthreads();
  for (int32_t s0 = 0; s0 < p.nseg; s0 += blockDim.x) {
    const int32_t s = s0 + threadIdx.x;
    unsigned long long range = 0, dense = 0;
    bool sat = false;
    if (s < p.nseg) {
      SegInfo& g = p.seg_info[s];
      const uint64_t npx = g.bx[1] >= 0 ? (uint64_t)((int64_t)g.bx[1] - g.bx[0] + 1) : 0;
      const uint64_t nnx = g.bx[2] < 0 ? (uint64_t)((int64_t)g.bx[3] - g.bx[2] + 1) : 0;
      const uint64_t npy = g.by[1] >= 0 ? (uint64_t)((int64_t)g.by[1] - g.by[0] + 1) : 0;
      const uint64_t nny = g.by[2] < 0 ? (uint64_t)((int64_t)g.by[3] - g.by[2] + 1) : 0;
      g.px = npx; g.wx = npx + nnx;
      g.py = npy; g.wy = npy + nny;
      g.ys = g.wy < 1 ? 1ull : g.wy;
      const int64_t npts = p.seg_off[s + 1] - p.seg_off[s];
      if (npts > 0) {
        // range = wx * ys, saturating (only one full-range cloud fits 64 bits)
        if (g.wx > (~0ull) / g.ys) { sat = true; range = ~0ull; }
        else range = g.wx * g.ys;
        const unsigned long long cap = (unsigned long long)(kDenseFactor * npts + kDenseSlack);
        if (!sat && range <= cap) dense = range;
        else atomicOr(&s_sparse, 1);
      }
    }
    s_range[threadIdx.x] = range;
    s_dense[threadIdx.x] = dense;
    if (sat && p.nseg > 1) atomicOr(&s_overflow, 1);
    __syncthreads();
    // Inclusive Hillis-Steele scan (saturating for ranges).
    for (int off = 1; off < (int)blockDim.x; off <<= 1) {
      unsigned long long r = 0, dn = 0;
      if ((int)threadIdx.x >= off) { r = s_range[threadIdx.x - off]; dn = s_dense[threadIdx.x - off]; }
      __syncthreads();
      if ((int)threadIdx.x >= off) {
        unsigned long long a = s_range[threadIdx.x];
        unsigned long long sum = a + r;
        if (sum < a) { sum = ~0ull; atomicOr(&s_overflow, 1); }
        s_range[threadIdx.x] = sum;
        s_dense[threadIdx.x] += dn;
      }
      __syncthreads();
    }
    if (s < p.nseg) {
      SegInfo& g = p.seg_info[s];
      const unsigned long long incl = s_range[threadIdx.x];
      unsigned long long base = s_carry_range + (incl - range);
      if (base < s_carry_range) atomicOr(&s_overflow, 1);
      g.base = base;
      g.map_base = dense > 0 ? (int64_t)(s_carry_dense + s_dense[threadIdx.x] - dense) : -1;
    }
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) {
      unsigned long long t = s_carry_range + s_range[threadIdx.x];
      if (t < s_carry_range) s_overflow = 1;
      s_carry_range = t;
      s_carry_dense += s_dense[threadIdx.x];
    }
    __syncthreads();
  }
  // Pooled budget: when the key ranges of all clouds together fit the dense
  // map (kDenseFactor * N + kDenseSlack per cloud, summed), every cloud gets
  // its slice of the map -- a cloud sparser than its own share borrows from
  // denser ones -- and the counting sort covers the whole batch: a cloud's
  // global key then equals its map index (map_base = base).
  __shared__ int s_pooled;
  if (threadIdx.x == 0)
    s_pooled = !p.force_radix && !s_overflow && s_carry_range <= (unsigned long long)p.dense_cap &&
               s_carry_range < (1ull << 31);
  __syncthreads();
  if (s_pooled) {
    for (int32_t s = threadIdx.x; s < p.nseg; s += blockDim.x) {
      SegInfo& g = p.seg_info[s];
      g.map_base = (int64_t)g.base;
    }
  }
  if (threadIdx.x == 0) {
    Desc* d = p.desc;
    // The last key is base[last] + range[last] - 1 (fits even when the sum
    // of ranges is exactly 2^64 for a single cloud).
    unsigned long long max_key = s_carry_range == 0 ? 0 : s_carry_range - 1;
    if (p.nseg == 1) {
      const SegInfo& g = p.seg_info[0];
      max_key = (g.wx == 0 || g.wy == 0) ? 0 : (g.wx - 1) * g.ys + (g.wy - 1);
    }
    uint32_t nbits = max_key == 0 ? 0 : 64 - __clzll((long long)max_key);
    uint32_t np = (nbits + kRadixBits - 1) / kRadixBits;
    d->nbits = nbits;
    d->npasses = np < 1 ? 1 : np;
    d->key64 = nbits > 32 ? 1 : 0;
    unsigned long long dt = s_pooled ? s_carry_range : s_carry_dense;
    if ((long long)dt > p.dense_cap) dt = 0;  // cannot happen by construction
    d->dense_total = dt;
    // Counting sort when the pooled map covers every cloud, or every
    // non-empty cloud is dense on its own (then the global key of a point is
    // its dense-map index too), and keys fit 31 bits.
    d->dense_sort = (s_pooled || (!p.force_radix && !s_sparse && !s_overflow && dt < (1ull << 31)))
                        ? 1u : 0u;
    if (s_overflow) set_error(d, kErrKeySpace);
  }
}

// ---------------------------------------------------------------- k_keys
// Points (keys) per thread whose loads are issued together in the key and
// count passes.
constexpr int kLoadBatch = 8;

// Compacted cell keys, one block per sort chunk, plus the chunk's histogram
// of the first digit (the count step of pass 0).
template <typename K>
__device__ __forceinline__ void keys_body(const Plan& p, uint32_t (*h)[kRadix]) {
  const int64_t n = p.n;
  K* keys = reinterpret_cast<K*>(p.keys[0]);
  const int64_t b0 = (int64_t)blockIdx.x * p.chunk_tiles * kSortTile;
  const int64_t b1 = min(n, b0 + (int64_t)p.chunk_tiles * kSortTile);
  const uint32_t warp = threadIdx.x >> 5;
  int32_t seg = b0 < b1 ? seg_of(p, b0) : 0;
  // kLoadBatch points per thread and round: their loads are in flight
  // together (a small cloud has few chunks, so each thread's rounds are the
  // kernel's critical path).
  for (int64_t i0 = b0 + threadIdx.x; i0 < b1; i0 += (int64_t)blockDim.x * kLoadBatch) {
    float2 v[kLoadBatch];
#pragma unroll
    for (int k = 0; k < kLoadBatch; ++k) {
      const int64_t i = i0 + (int64_t)k * blockDim.x;
      if (i < b1) v[k] = p.X[i];
    }
#pragma unroll
    for (int k = 0; k < kLoadBatch; ++k) {
      const int64_t i = i0 + (int64_t)k * blockDim.x;
      if (i < b1) {
        while (i >= p.seg_off[seg + 1]) ++seg;
        const SegInfo& g = p.seg_info[seg];
        const float inv_r = p.seg_param[seg].inv_r;
        const uint64_t gx = compact_axis(cell_coord(v[k].x, inv_r), g.bx, g.px);
        const uint64_t gy = compact_axis(cell_coord(v[k].y, inv_r), g.by, g.py);
        const uint64_t key = g.base + gx * g.ys + gy;
        keys[i] = (K)key;
        atomicAdd(&h[warp][key & (kRadix - 1)], 1u);
      }
    }
  }
}

__global__ void __launch_bounds__(kSortThreads) k_keys(Plan p) {
  __shared__ uint32_t h[kSortWarps][kRadix];
  Desc* d = p.desc;
  if (d->dense_sort) return;
  for (int i = threadIdx.x; i < kSortWarps * kRadix; i += blockDim.x) (&h[0][0])[i] = 0;
  __syncthreads();
  if (d->key64) keys_body<uint64_t>(p, h);
  else keys_body<uint32_t>(p, h);
  __syncthreads();
  {
    const uint32_t t = threadIdx.x;
    uint32_t sum = 0;
#pragma unroll
    for (int w = 0; w < kSortWarps; ++w) sum += h[w][t];
    p.chunk_count[(int64_t)t * p.sort_chunks + blockIdx.x] = sum;
    if (sum) atomicAdd(&d->digit_total[0][t], sum);
  }
  // Clearing duties for later kernels (their look-back words and the dense
  // cell map must start empty).
  const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t dense = (int64_t)d->dense_total;
  for (int64_t i = tid; i < dense; i += stride) p.cell_map[i] = -1;
}

// ------------------------------------------------------- radix sort kernel
// The LSD sort for key spaces too wide for the counting sort (and for the
// debug entry point, whose perm must be stable): one cooperative kernel runs
// every pass the device-side pass count asks for, each pass as three phases
// separated by grid barriers (no unused passes, no extra launches):
//   count    histogram of the digit per chunk (pass 0: done by k_keys)
//   scan     per digit, exclusive scan of its row of chunk counts, offset by
//            the total of all lower digits
//   scatter  each chunk, tile by tile: stable ranking of 4096 keys in shared
//            memory, staged scatter so each digit run is written
//            contiguously; the last pass writes perm and gathers the sorted
//            float2 coordinates
template <typename K>
__device__ __forceinline__ void count_body(const Plan& p, int pass, int32_t chunk, uint32_t (*h)[kRadix]) {
  const int64_t n = p.n;
  const K* keys = reinterpret_cast<const K*>(p.keys[pass & 1]);
  const int64_t b0 = (int64_t)chunk * p.chunk_tiles * kSortTile;
  const int64_t b1 = min(n, b0 + (int64_t)p.chunk_tiles * kSortTile);
  const uint32_t shift = pass * kRadixBits;
  const uint32_t warp = threadIdx.x >> 5;
  for (int i = threadIdx.x; i < kSortWarps * kRadix; i += blockDim.x) (&h[0][0])[i] = 0;
  __syncthreads();
  for (int64_t i0 = b0 + threadIdx.x; i0 < b1; i0 += (int64_t)blockDim.x * kLoadBatch) {
    K kk[kLoadBatch];
#pragma unroll
    for (int k = 0; k < kLoadBatch; ++k) {
      const int64_t i = i0 + (int64_t)k * blockDim.x;
      kk[k] = i < b1 ? keys[i] : (K)0;
    }
#pragma unroll
    for (int k = 0; k < kLoadBatch; ++k)
      if (i0 + (int64_t)k * blockDim.x < b1)
        atomicAdd(&h[warp][(uint32_t)((uint64_t)kk[k] >> shift) & (kRadix - 1)], 1u);
  }
  __syncthreads();
  const uint32_t t = threadIdx.x;
  uint32_t sum = 0;
#pragma unroll
  for (int w = 0; w < kSortWarps; ++w) sum += h[w][t];
  p.chunk_count[(int64_t)t * p.sort_chunks + chunk] = sum;
  if (sum) atomicAdd(&p.desc->digit_total[pass & 1][t], sum);
  __syncthreads();
}

// Exclusive scan of digit `dig`'s row of chunk counts (sort_chunks <=
// kMaxChunks = 4 * kSortThreads entries), offset by the total of the lower
// digits.
__device__ __forceinline__ void scan_body(const Plan& p, int pass, uint32_t dig, uint32_t* s_warp) {
  Desc* d = p.desc;
  const uint32_t lane = lane_id(), warp = threadIdx.x >> 5;
  uint32_t base = 0;
  for (uint32_t t = lane; t < dig; t += 32) base += d->digit_total[pass & 1][t];
  base = __reduce_add_sync(0xffffffffu, base);
  uint32_t* row = p.chunk_count + (int64_t)dig * p.sort_chunks;
  const int32_t b0 = threadIdx.x * 4;
  uint32_t v[4], sum = 0;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    v[k] = b0 + k < p.sort_chunks ? row[b0 + k] : 0u;
    sum += v[k];
  }
  uint32_t x = sum;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= (uint32_t)o) x += y;
  }
  if (lane == 31) s_warp[warp] = x;
  __syncthreads();
  uint32_t run = base + x - sum;
  for (uint32_t w = 0; w < warp; ++w) run += s_warp[w];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    if (b0 + k < p.sort_chunks) row[b0 + k] = run;
    run += v[k];
  }
  __syncthreads();
}

// The same scan by one warp, for rows of at most kWarpScanChunks chunk
// counts (4 per lane): a block scans kSortWarps digits at once, so a small
// grid covers all kRadix digits in one step.
constexpr int kWarpScanChunks = 128;

__device__ __forceinline__ void scan_warp(const Plan& p, int pass, uint32_t dig) {
  Desc* d = p.desc;
  const uint32_t lane = lane_id();
  uint32_t base = 0;
  for (uint32_t t = lane; t < dig; t += 32) base += d->digit_total[pass & 1][t];
  base = __reduce_add_sync(0xffffffffu, base);
  uint32_t* row = p.chunk_count + (int64_t)dig * p.sort_chunks;
  const int32_t b0 = lane * 4;
  uint32_t v[4], sum = 0;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    v[k] = b0 + k < p.sort_chunks ? row[b0 + k] : 0u;
    sum += v[k];
  }
  uint32_t x = sum;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= (uint32_t)o) x += y;
  }
  uint32_t run = base + x - sum;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    if (b0 + k < p.sort_chunks) row[b0 + k] = run;
    run += v[k];
  }
}

__device__ __forceinline__ uint32_t digit_of(uint32_t key, uint32_t shift) {
  return (key >> shift) & (kRadix - 1);
}
__device__ __forceinline__ uint32_t digit_of(uint64_t key, uint32_t shift) {
  return (uint32_t)(key >> shift) & (kRadix - 1);
}

struct SweepSmem {
  uint32_t wcnt[kSortWarps][kRadix + 1];  // per-warp digit counts -> warp offsets
                                          // (slot kRadix absorbs invalid items)
  uint32_t tile_excl[kRadix];          // exclusive scan of tile digit counts
  uint32_t glob[kRadix];               // output position of this tile's digit runs
  uint32_t carry[kRadix];              // next output position of each digit
  uint32_t warp_tot[kSortWarps];
  uint32_t warp_tot_wide[kSortWarps];
  __device__ uint32_t (*wcnt_as_hist())[kRadix] {
    return reinterpret_cast<uint32_t (*)[kRadix]>(&wcnt[0][0]);
  }
};

template <typename K>
__device__ __forceinline__ void scatter_body(const Plan& p, int pass, bool last, int32_t chunk,
                                             SweepSmem& sm, unsigned char* stage_raw) {
  const int64_t n = p.n;
  const uint32_t lane = lane_id();
  const uint32_t warp = threadIdx.x >> 5;
  const uint32_t shift = pass * kRadixBits;
  const int src = pass & 1;
  const K* keys_in = reinterpret_cast<const K*>(p.keys[src]);
  K* keys_out = reinterpret_cast<K*>(p.keys[src ^ 1]);
  const uint32_t* vals_in = p.vals[src];
  uint32_t* vals_out = last ? p.perm : p.vals[src ^ 1];
  K* st_keys = reinterpret_cast<K*>(stage_raw);
  uint32_t* st_vals = reinterpret_cast<uint32_t*>(stage_raw + sizeof(K) * kSortTile);

  sm.carry[threadIdx.x] = p.chunk_count[(int64_t)threadIdx.x * p.sort_chunks + chunk];
  const int64_t c0 = (int64_t)chunk * p.chunk_tiles * kSortTile;
  const int64_t c1 = min(n, c0 + (int64_t)p.chunk_tiles * kSortTile);
  for (int64_t tile_base = c0; tile_base < c1; tile_base += kSortTile) {
    for (int i = threadIdx.x; i < kSortWarps * (kRadix + 1); i += blockDim.x) (&sm.wcnt[0][0])[i] = 0;
    __syncthreads();
    const int64_t wbase = tile_base + (int64_t)warp * 32 * kSortItems;
    // Keys of this warp's slice in (k, lane) order; digits are recomputed
    // and values read at staging time to keep few registers live.
    K key[kSortItems];
    uint32_t rank[kSortItems];
#pragma unroll
    for (int k = 0; k < kSortItems; ++k) {
      const int64_t gi = wbase + k * 32 + lane;
      key[k] = gi < c1 ? keys_in[gi] : (K)0;
    }
    // Stable warp ranking in (k, lane) order. Peers (lanes holding the same
    // digit) come from one ballot per digit bit; the first lane of each peer
    // group advances the warp's counter for the digit.
    const uint32_t lt = lanemask_lt();
#pragma unroll
    for (int k = 0; k < kSortItems; ++k) {
      const int64_t gi = wbase + k * 32 + lane;
      const bool valid = gi < c1;
      const uint32_t dk = digit_of(key[k], shift);
      uint32_t peers = __ballot_sync(0xffffffffu, valid);
      if (!valid) peers = ~peers;
#pragma unroll
      for (int b = 0; b < kRadixBits; ++b) {
        const bool bit = (dk >> b) & 1u;
        const uint32_t m = __ballot_sync(0xffffffffu, bit);
        peers &= bit ? m : ~m;
      }
      const uint32_t slot = valid ? dk : (uint32_t)kRadix;
      const uint32_t pre = __popc(peers & lt);
      const uint32_t old = sm.wcnt[warp][slot];
      __syncwarp();
      if (pre == 0) sm.wcnt[warp][slot] = old + __popc(peers);
      __syncwarp();
      rank[k] = old + pre;
    }
    __syncthreads();
    {
      const uint32_t t = threadIdx.x;
      uint32_t run = 0;
#pragma unroll
      for (int w = 0; w < kSortWarps; ++w) {
        const uint32_t c = sm.wcnt[w][t];
        sm.wcnt[w][t] = run;
        run += c;
      }
      uint32_t x = run;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= (uint32_t)o) x += y;
      }
      if (lane == 31) sm.warp_tot[warp] = x;
      __syncthreads();
      uint32_t wpre = 0;
      for (uint32_t w = 0; w < warp; ++w) wpre += sm.warp_tot[w];
      sm.tile_excl[t] = wpre + x - run;
      sm.glob[t] = sm.carry[t];
      sm.carry[t] += run;
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < kSortItems; ++k) {
      const int64_t gi = wbase + k * 32 + lane;
      if (gi < c1) {
        const uint32_t dk = digit_of(key[k], shift);
        const uint32_t lp = sm.tile_excl[dk] + sm.wcnt[warp][dk] + rank[k];
        st_keys[lp] = key[k];
        st_vals[lp] = pass == 0 ? (uint32_t)gi : vals_in[gi];
      }
    }
    __syncthreads();
    const int32_t valid = (int32_t)min((int64_t)kSortTile, c1 - tile_base);
    for (int32_t lp = threadIdx.x; lp < valid; lp += blockDim.x) {
      const K kk = st_keys[lp];
      const uint32_t dk = digit_of(kk, shift);
      const uint32_t gpos = sm.glob[dk] + (uint32_t)lp - sm.tile_excl[dk];
      const uint32_t vv = st_vals[lp];
      keys_out[gpos] = kk;
      vals_out[gpos] = vv;
    }
    __syncthreads();
  }
}

__global__ void __launch_bounds__(kSortThreads, 3) k_radix(Plan p) {
  extern __shared__ __align__(16) unsigned char dyn_smem[];
  SweepSmem& sm = *reinterpret_cast<SweepSmem*>(dyn_smem);
  unsigned char* stage = dyn_smem + ((sizeof(SweepSmem) + 15) & ~size_t(15));
  Desc* d = p.desc;
  if (d->dense_sort) return;
  const int np = (int)d->npasses;
  const bool wide = d->key64 != 0;
  for (int pass = 0; pass < np; ++pass) {
    if (pass > 0) {
      for (int32_t ch = blockIdx.x; ch < p.sort_chunks; ch += gridDim.x) {
        if (wide) count_body<uint64_t>(p, pass, ch, sm.wcnt_as_hist());
        else count_body<uint32_t>(p, pass, ch, sm.wcnt_as_hist());
      }
      grid_sync(&d->bar, d);
    }
    if (p.sort_chunks <= kWarpScanChunks) {
      for (uint32_t dig = blockIdx.x * kSortWarps + (threadIdx.x >> 5); dig < (uint32_t)kRadix;
           dig += gridDim.x * kSortWarps)
        scan_warp(p, pass, dig);
    } else {
      for (uint32_t dig = blockIdx.x; dig < (uint32_t)kRadix; dig += gridDim.x)
        scan_body(p, pass, dig, sm.warp_tot_wide);
    }
    if (blockIdx.x == 0)
      for (int t = threadIdx.x; t < kRadix; t += blockDim.x) d->digit_total[(pass & 1) ^ 1][t] = 0;
    grid_sync(&d->bar, d);
    const bool last = pass == np - 1;
    for (int32_t ch = blockIdx.x; ch < p.sort_chunks; ch += gridDim.x) {
      if (wide) scatter_body<uint64_t>(p, pass, last, ch, sm, stage);
      else scatter_body<uint32_t>(p, pass, last, ch, sm, stage);
    }
    if (pass + 1 < np) grid_sync(&d->bar, d);
  }
}

constexpr size_t kSweepSmemBytes =
    ((sizeof(SweepSmem) + 15) & ~size_t(15)) + (sizeof(uint64_t) + sizeof(uint32_t)) * kSortTile;

// ------------------------------------------------------------- launchers
static int grid_for(const Plan& p, int64_t work, int threads, int per_sm) {
  int64_t g = (work + threads - 1) / threads;
  const int64_t cap = (int64_t)p.num_sms * per_sm;
  if (g > cap) g = cap;
  if (g < 1) g = 1;
  return (int)g;
}

cudaError_t launch_front(const Plan& p, cudaStream_t s) {
  k_init<<<grid_for(p, (int64_t)p.nseg + p.ids_tiles + 2 * kRadix, 256, 2), 256, 0, s>>>(p);
  k_bounds<<<grid_for(p, p.n, 256 * 8, 8), 256, 0, s>>>(p);
  // One block; its scans take log2(threads) rounds of block barriers, so a
  // call with few clouds takes a small block (one warp for a plain call).
  const int fin_threads = p.nseg <= 32 ? 32 : (p.nseg <= 256 ? 256 : 1024);
  k_seg_finalize<<<1, fin_threads, 0, s>>>(p);
  return cudaGetLastError();
}

cudaError_t launch_keys(const Plan& p, cudaStream_t s) {
  k_keys<<<p.sort_chunks, kSortThreads, 0, s>>>(p);
  return cudaGetLastError();
}

// Cooperative launch: every block of the grid must be resident for the grid
// barriers. One block per sort chunk (the count and scatter phases loop over
// chunks), within the occupancy-derived number of resident blocks.
cudaError_t launch_radix(const Plan& p, cudaStream_t s) {
  static PerDeviceBlocks cache;
  int blocks_per_sm = 0;
  cudaError_t e = cache.get(
      [](int* b) {
        cudaError_t r = cudaFuncSetAttribute(k_radix, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)kSweepSmemBytes);
        if (r != cudaSuccess) return r;
        return cudaOccupancyMaxActiveBlocksPerMultiprocessor(b, k_radix, kSortThreads, kSweepSmemBytes);
      },
      &blocks_per_sm);
  if (e != cudaSuccess) return e;
  const int grid = coop_grid(p.sort_chunks, p.num_sms, p.num_sms * blocks_per_sm);
  Plan q = p;
  void* args[] = {&q};
  return cudaLaunchCooperativeKernel((const void*)k_radix, dim3(grid), dim3(kSortThreads), args,
                                     kSweepSmemBytes, s);
}

}  // namespace dbs
