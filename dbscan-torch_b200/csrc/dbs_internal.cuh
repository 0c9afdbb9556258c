// dbs_internal.cuh -- shared types and device helpers of the sm_100a DBSCAN
// pipeline. Not part of the public C-ABI (include/dbscan_b200.h).
//
// Pipeline (one stream, no host synchronisation; every count that sizes a
// loop lives in device memory, so the whole sequence can be captured in a
// CUDA graph):
//
//   k_init         zero per-call counters, histograms, per-cloud bounds
//   k_bounds       per-cloud bounds of the cell coordinates (kx, ky)
//   k_seg_finalize per-cloud compacted key ranges, key bases, sort form
//   k_csort        dense key spaces: counting sort, cells, dense cell map
//   k_keys, k_radix  otherwise: keys + LSD radix sort (return at once when
//                  the counting sort ran, and k_csort returns when they run)
//   k_rle          run-length cells after the radix sort
//   k_cell_prep    per-cell box + 25-entry neighbour row; point classes
//   k_core         core flags of the query points
//   k_status       cell status, union-find init
//   k_pairs / k_pair_scan / k_pair_warp (two rings, k_flatten between)
//                  cell-graph union-find over core cells
//   k_ids          flatten + exclusive scan of root flags (look-back)
//   k_cid          cluster id per cell
//   k_labels       border assignment, core labels, unpermute
//
// The plain call is the batched call with one cloud: every kernel works on
// a segmented layout (clouds concatenated, each with its own eps and
// min_samples, disjoint key ranges).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>

namespace dbs {

constexpr int kRadixBits = 8;
constexpr int kRadix = 1 << kRadixBits;
constexpr int kMaxPasses = 64 / kRadixBits;
constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kSortItems = 16;
constexpr int kSortTile = kSortThreads * kSortItems;
constexpr int kMaxChunks = 1024;
constexpr int kMaxGrid = 4096;   // blocks of a cooperative launch (bound)
constexpr int kScanThreads = 256;
constexpr int kScanItems = 16;
constexpr int kScanTile = kScanThreads * kScanItems;
constexpr int kIdsItems = 8;                    // cells per lane of a k_ids tile
constexpr int kIdsTile = kScanThreads * kIdsItems;
constexpr int kCellThreads = 256;               // warp-per-cell kernels
constexpr uint32_t kSpinCap = 1u << 22;         // bounded waits (look-back polls)
constexpr uint32_t kFindCap = 1u << 20;         // bounded union-find walks / retries
constexpr uint32_t kBarrierCap = 1u << 18;      // bounded grid-barrier polls (~0.1 s)
constexpr int kNgh = 25;
constexpr int32_t kHugeCell = 4096;   // cells whose box is reduced by many warps
constexpr int32_t kHugeChunk = 2048;  // points per chunk of a huge cell

// Dense cell map: a cloud whose compacted key range W satisfies
// W <= kDenseFactor * N + kDenseSlack resolves neighbours with one load; a
// batch whose clouds' ranges fit the summed budget gets a map for every
// cloud (k_seg_finalize).
constexpr int64_t kDenseFactor = 6;
// Counting sort: a key that at least kHotGroup lanes of one 32-point row
// share is hot; up to kHotSlots hot keys get their points ranked by the count
// pass instead of a second fetch-add in the scatter.
constexpr int kHotSlots = 64;
constexpr uint32_t kHotGroup = 8;
constexpr int64_t kDenseSlack = 4096;

// Grid-stride kernels whose grid (blocks per SM) a launch shape may set
// (dbs_launch_shape of the C-ABI, same indices), and their built-in grids.
// The label pass takes 32 blocks per SM while its border items go first
// (n <= kCoreFirstPoints): they scan uneven numbers of neighbour points, and
// smaller grid-stride shares balance them (10M constant-density points: 0.843
// against 0.855 ms per call with 8). With the core items first (more points)
// 8 blocks per SM is faster (4,096-cloud batch, 151M points: 22.1 against
// 22.9 ms with 32).
enum : int {
  kTuneCount = 0,
  kTuneCellPrep,
  kTuneCore,
  kTunePairs,
  kTunePairScan,
  kTuneLabels,
  kNumTuned
};
// The count kernel's launch bounds let 6 blocks per SM be resident; a grid of
// exactly those (no second partial wave) measured 76.0 -> 71.8 us at 10M
// points and 456 -> 349 us on a 1,024-cloud batch. The cell pass keeps 8 (5
// are resident) though: 5 measured 106.9 -> 121.7 us at 10M points.
constexpr int32_t kDefaultBlocksPerSm[kNumTuned] = {6, 8, 8, 8, 8, 8};
constexpr int32_t kLabelsBlocksPerSmBorderFirst = 32;
// Runs of up to this many points take the latency-bound forms of the cell,
// core and label passes (wider groups of independent loads, several lanes
// per cell); larger runs take the forms that keep more warps resident.
constexpr int64_t kSmallRun = 2 << 20;
// Label pass item order: border items first up to this many points (labels
// that fit L2), core items first above (k_labels).
constexpr int64_t kCoreFirstPoints = 16 << 20;
// Built-in blocks per SM of tuned kernel k for a run over n points.
inline int32_t default_blocks_per_sm(int k, int64_t n) {
  if (k == kTuneLabels && n <= kCoreFirstPoints) return kLabelsBlocksPerSmBorderFirst;
  return kDefaultBlocksPerSm[k];
}

// Error bits of Desc::status (OR-ed by kernels, read by the host).
enum : uint32_t {
  kErrLookback = 1u << 0,   // a decoupled look-back wait hit its cap
  kErrFind = 1u << 1,       // a union-find walk / hook loop hit its cap
  kErrKeySpace = 1u << 2,   // batched key ranges overflow 64 bits
  kErrBarrier = 1u << 3,    // a grid barrier wait hit its cap
  kErrCapacity = 1u << 4,   // a work list overflowed, or a sorted position out of range
};

// Dynamic work counters (Desc::ctr).
enum : int {
  kCtrRle = 0,
  kCtrPrep,
  kCtrCore,
  kCtrIds,
  kCtrLabels,
  kCtrBig,
  kCtrDebug,
  kNumCtr
};

// Host-computed per-cloud scalars (dbscan_cuda.cu:547-550 of the reference:
// fl_eps = (float)eps, inv_r = sqrtf(2)/fl_eps, eps_sq = fl_eps*fl_eps on
// the host in IEEE float, ms = (int32)min_samples).
struct SegParam {
  float inv_r;
  float eps_sq;
  int32_t ms;
  int32_t pad;
};

// Device-computed per-cloud layout. Cell coordinates are split into the
// non-negative and negative classes so that the compaction preserves the
// reference's unsigned key order ((u32)kx << 32 | (u32)ky): non-negative
// coordinates come first, then negative ones, each class ascending.
// The compacted key of cell (gx, gy) is base + gx * wy + gy (mixed radix,
// no padding of the y width to a power of two): lexicographic in (gx, gy),
// and a cell's coordinates come back from its key with a division by wy.
struct SegInfo {
  int32_t bx[4];     // x: lo_pos, hi_pos, lo_neg, hi_neg (atomics)
  int32_t by[4];     // y: same
  uint64_t px, wx;   // x: width of the non-negative class, total width
  uint64_t py, wy;   // y: same
  uint64_t base;     // first global key of this cloud
  int64_t map_base;  // offset in the dense cell map, -1 when not dense
  int32_t cell_begin;  // first cell index of this cloud (filled by k_rle)
  uint64_t ys;       // key stride of one x column: max(wy, 1)
};

// Software grid barrier of the cooperative kernels (all blocks resident).
struct GridBar {
  unsigned int count;
  unsigned int gen;
};

struct Desc {
  uint32_t status;
  uint32_t key64;      // keys stored as u64 (else u32)
  uint32_t nbits;      // significant key bits
  uint32_t npasses;    // radix passes that run (>= 1)
  uint32_t num_cells;
  uint32_t pad0;
  uint64_t dense_total;  // dense-map entries in use
  unsigned long long big_packed;  // huge cells: entries << 40 | chunks
  uint32_t ctr[kNumCtr];
  uint32_t digit_total[2][kRadix];  // per-pass digit totals (ping-pong)
  uint32_t dense_sort;  // 1: counting sort over the dense key space
  uint32_t q_count;     // core-query list length (points of cells below ms)
  uint32_t b_count;     // border list length (non-core points)
  uint32_t p_count;     // union-find candidate pair list length
  uint32_t d_count;     // pairs deferred to warp-cooperative scans
  uint32_t hot_used;    // counting sort: occupied hot-key slots
  uint32_t ring_pairs[2];  // p_count of each union pass (kept for the stats read-back)
  uint32_t ring_warp[2];   // d_count of each union pass
  GridBar bar;
  // %globaltimer (ns) at each phase boundary of the cooperative kernels,
  // written by block 0 after each grid barrier: a per-phase split readable
  // from the workspace without a profiler.
  unsigned long long phase_ns[16];
};

// Device pointers of one call, carved out of the caller's workspace.
struct Plan {
  Desc* desc;
  const float2* X;        // (n) input points, AoS
  int32_t* labels;        // (n) output labels, input order
  int64_t* seg_off;       // (nseg+1)
  SegParam* seg_param;    // (nseg)
  SegInfo* seg_info;
  void* keys[2];          // ping-pong key buffers (u32 or u64 elements)
  uint32_t* vals[2];      // ping-pong index buffers
  uint32_t* perm;         // (n) sorted position -> input index
  float2* xy;             // (n) sorted coordinates
  uint8_t* is_core;       // (n) sorted order
  uint32_t* chunk_count;  // (kRadix * sort_chunks) digit-major counts / offsets
  unsigned long long* rle_status;
  unsigned long long* ids_status;
  int32_t* point_cell;    // (n) cell of each sorted point
  int32_t* cell_start;    // (n+1)
  uint64_t* cell_key;     // (n)
  int32_t* cell_seg;      // (n)
  float4* bbox;           // (n) xmin, xmax, ymin, ymax
  int32_t* ngh;           // (n*25)
  uint8_t* cell_status;   // (n) 0 none, 1 mixed, 2 all core
  int32_t* uf;            // (n)
  int32_t* root_rank;     // (n) exclusive scan of root flags
  int32_t* cid;           // (n) cluster id per cell
  uint32_t* qlist;        // (n) sorted positions needing a core count
  uint32_t* blist;        // (n) sorted positions of non-core points
  int2* plist;            // (pair_cap) candidate cell pairs (c, nc > c)
  uint32_t* dlist;        // (pair_cap) indices into plist, over budget
  int64_t pair_cap;       // entries available in plist / dlist
  int32_t* cell_map;      // dense cell map
  int64_t dense_cap;      // entries available in cell_map
  int32_t* big_cell;      // huge cells (> kHugeCell points): cell index
  unsigned long long* big_base;  // first chunk of each huge cell
  uint32_t* big_done;     // chunks finished per huge cell
  float4* big_chunk_box;  // bounding box of each chunk
  int64_t big_cap;        // entries available in big_cell
  int64_t chunk_cap;      // entries available in big_chunk_box
  uint32_t* bin_count;    // counting sort: per-key counts -> offsets -> cursors
  uint32_t* blk_sum;      // counting sort: per-block bin sums (kMaxGrid)
  uint32_t* blk_ne;       // counting sort: per-block non-empty bin counts
  uint32_t* hot_key;      // counting sort: hot-key table (kHotSlots each)
  uint32_t* hot_cnt;      //   points of hot rows per hot key
  uint32_t* hot_cold;     //   points of the key outside hot rows
  uint32_t* hot_base;     //   first sorted position of the key's hot points
  int32_t force_radix;    // debug entry: stable radix sort (reference perm)
  int64_t n;
  int32_t nseg;
  int32_t sort_chunks;    // chunks of the radix passes (one block each)
  int32_t chunk_tiles;    // kSortTile tiles per chunk
  int32_t scan_tiles;     // ceil(n / kScanTile)
  int32_t ids_tiles;      // ceil(n / kIdsTile)
  int32_t num_sms;
  int32_t bps[kNumTuned]; // blocks per SM of the tuned kernels
  int32_t single;         // one cloud: k_init writes seg_off / seg_param
  SegParam single_param;
};

// ------------------------------------------------------------- device math
// Every operation below is IEEE round-to-nearest with subnormals flushed
// (the library is compiled with -ftz=true -fmad=false), matching the
// reference build's --use_fast_math arithmetic on the values it produces.
__device__ __forceinline__ float sq_dist(float ex, float ey) {
  // fma(ex, ex, ey*ey): the contraction of `ex*ex + ey*ey` found in the
  // reference build at every call site.
  return __fmaf_rn(ex, ex, __fmul_rn(ey, ey));
}

// dbscan_cuda.cu:183-187
__device__ __forceinline__ float point_box_d2(float x, float y, float4 b) {
  float dx = fmaxf(fmaxf(__fsub_rn(b.x, x), __fsub_rn(x, b.y)), 0.0f);
  float dy = fmaxf(fmaxf(__fsub_rn(b.z, y), __fsub_rn(y, b.w)), 0.0f);
  return sq_dist(dx, dy);
}

// Largest squared distance from (x, y) to a point of box b, in the same
// rounded form as the pairwise test: every fsub and the fma are monotone in
// the magnitudes of their operands, so for any point p inside b,
// d2(p, (x, y)) <= point_box_max_d2(x, y, b). A cell whose box passes
// `<= eps_sq` therefore has every point within eps (cells holding a NaN
// coordinate carry an infinite box, which never passes).
__device__ __forceinline__ float point_box_max_d2(float x, float y, float4 b) {
  const float dx = fmaxf(fabsf(__fsub_rn(b.x, x)), fabsf(__fsub_rn(b.y, x)));
  const float dy = fmaxf(fabsf(__fsub_rn(b.z, y)), fabsf(__fsub_rn(b.w, y)));
  return sq_dist(dx, dy);
}

// dbscan_cuda.cu:190-194
__device__ __forceinline__ float box_box_d2(float4 a, float4 b) {
  float dx = fmaxf(fmaxf(__fsub_rn(b.x, a.y), __fsub_rn(a.x, b.y)), 0.0f);
  float dy = fmaxf(fmaxf(__fsub_rn(b.z, a.w), __fsub_rn(a.z, b.w)), 0.0f);
  return sq_dist(dx, dy);
}

// (int32)floorf(v): round toward -inf, saturating, NaN -> 0.
__device__ __forceinline__ int32_t cell_coord(float v, float inv_r) {
  return __float2int_rd(__fmul_rn(v, inv_r));
}

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }

__device__ __forceinline__ uint32_t lanemask_lt() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// Segment (cloud) of input/sorted position i. Points of a cloud are
// contiguous in input order and, because cloud key ranges are disjoint and
// ascending, in sorted order too.
__device__ __forceinline__ int32_t seg_of(const Plan& p, int64_t i) {
  if (p.nseg == 1) return 0;
  int32_t lo = 0, hi = p.nseg - 1;
  while (lo < hi) {
    int32_t mid = (lo + hi + 1) >> 1;
    if (p.seg_off[mid] <= i) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// Compacted coordinate of kx along one axis, or -1 (as u64 ~0) when the
// coordinate is outside the cloud's occupied classes.
__device__ __forceinline__ uint64_t compact_axis(int32_t k, const int32_t b[4], uint64_t pw) {
  if (k >= 0) {
    if (b[1] < 0 || k < b[0] || k > b[1]) return ~0ull;
    return (uint64_t)(uint32_t)(k - b[0]);
  }
  if (b[2] == 0 || k < b[2] || k > b[3]) return ~0ull;
  return pw + (uint64_t)(uint32_t)(k - b[2]);
}

// Cloud owning global key b: the last cloud whose key base is <= b (empty
// clouds share their base with the next cloud and come before it).
__device__ __forceinline__ int32_t seg_of_key(const Plan& p, uint64_t b) {
  if (p.nseg == 1) return 0;
  int32_t lo = 0, hi = p.nseg - 1;
  while (lo < hi) {
    const int32_t mid = (lo + hi + 1) >> 1;
    if (p.seg_info[mid].base <= b) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// Per-cloud scalars of the dense key of a point (its dense-map index, which
// fits 31 bits), held in registers while a thread's points stay in one cloud.
struct KeyCtx {
  int32_t bx[4], by[4];
  uint64_t px, py, base, ys;
  float inv_r;
  int64_t end;  // first input index past the cloud
  int32_t seg;
  __device__ void load(const Plan& p, int32_t s) {
    const SegInfo& g = p.seg_info[s];
#pragma unroll
    for (int k = 0; k < 4; ++k) { bx[k] = g.bx[k]; by[k] = g.by[k]; }
    px = g.px; py = g.py; base = g.base; ys = g.ys;
    inv_r = p.seg_param[s].inv_r;
    end = p.seg_off[s + 1];
    seg = s;
  }
  __device__ uint32_t key(float2 v) const {
    const uint64_t gx = compact_axis(cell_coord(v.x, inv_r), bx, px);
    const uint64_t gy = compact_axis(cell_coord(v.y, inv_r), by, py);
    return (uint32_t)(base + gx * ys + gy);
  }
};

__device__ __forceinline__ void set_error(Desc* d, uint32_t bits) {
  atomicOr(&d->status, bits);
}


// Relaxed device-scope 64-bit load/store for look-back words.
__device__ __forceinline__ unsigned long long ld_relaxed(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_relaxed(unsigned long long* p, unsigned long long v) {
  asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" :: "l"(p), "l"(v) : "memory");
}

constexpr unsigned long long kFlagAgg = 1ull << 62;
constexpr unsigned long long kFlagInc = 2ull << 62;
constexpr unsigned long long kValMask = (1ull << 62) - 1;

// Decoupled look-back over look-back words laid out with `stride` between
// consecutive tiles, walked by a whole warp (all 32 lanes call it with the
// same arguments); returns the exclusive prefix of tile `tile`. Each round
// reads the 32 nearest unconsumed predecessors at once, consumes them up to
// the first one not yet published and stops at the first inclusive prefix,
// so a walk over many published aggregates costs one round trip per 32
// tiles. Bounded: a wait that exceeds kSpinCap polls sets kErrLookback and
// gives up.
__device__ __forceinline__ unsigned long long lookback_warp(const unsigned long long* words,
                                                            int64_t tile, int64_t stride, Desc* d) {
  const uint32_t full = 0xffffffffu;
  const int lane = (int)(threadIdx.x & 31u);
  unsigned long long excl = 0;
  int64_t j = tile - 1;  // nearest predecessor not consumed yet
  uint32_t spins = 0;
  while (j >= 0) {
    const int64_t idx = j - lane;
    // Before tile 0 there is nothing: an inclusive prefix of zero.
    const unsigned long long v = idx >= 0 ? ld_relaxed(words + idx * stride) : kFlagInc;
    const unsigned long long flag = v & ~kValMask;
    const uint32_t not_ready = __ballot_sync(full, flag == 0);
    const uint32_t inclusive = __ballot_sync(full, flag == kFlagInc);
    const int first_nr = not_ready ? __ffs(not_ready) - 1 : 32;
    const int first_inc = inclusive ? __ffs(inclusive) - 1 : 32;
    const bool done = first_inc < first_nr;
    const int take = done ? first_inc + 1 : first_nr;  // lanes [0, take) are consumed
    unsigned long long part = lane < take ? (v & kValMask) : 0ull;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(full, part, o);
    excl += part;
    if (done) return excl;
    j -= take;
    if (take < 32 && ++spins > kSpinCap) {
      set_error(d, kErrLookback);
      break;
    }
  }
  return excl;
}

__device__ __forceinline__ unsigned int ld_acquire_u32(const unsigned int* p) {
  unsigned int v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Grid-wide barrier for cooperative launches. Bounded: a wait past
// kSpinCap polls sets kErrBarrier and returns (the kernel then finishes with
// invalid results rather than hanging).
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void mark_phase(Desc* d, int k) {
  if (blockIdx.x == 0 && threadIdx.x == 0 && k < 16) d->phase_ns[k] = global_ns();
}

__device__ __forceinline__ void grid_sync(GridBar* b, Desc* d) {
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned int g = ld_acquire_u32(&b->gen);
    __threadfence();
    if (atomicAdd(&b->count, 1u) == gridDim.x - 1) {
      atomicExch(&b->count, 0u);
      __threadfence();
      atomicAdd(&b->gen, 1u);
    } else {
      uint32_t spins = 0;
      while (ld_acquire_u32(&b->gen) == g) {
        if (++spins > kBarrierCap) { set_error(d, kErrBarrier); break; }
        __nanosleep(64);
      }
    }
    __threadfence();
  }
  __syncthreads();
}

// --------------------------------------------------------- host launchers
// One-time set-up of a cooperative kernel on the current device (dynamic
// shared-memory attribute, resident blocks per SM). Kernel attributes belong
// to a device, so the result is cached per device ordinal: a process that
// runs on cuda:0 and then on cuda:1 sets the attribute on both. `setup(&b)`
// sets the attributes and stores the resident blocks per SM in b. The mutex
// serialises host threads that launch at the same time.
constexpr int kMaxDevices = 64;
// Grid of a cooperative kernel: `want` blocks for its work, at least one
// block per SM, at most the resident blocks (every block of a cooperative
// launch must be resident). A grid barrier costs one atomic per block on one
// counter plus the wait for the last block, so a run with little work keeps
// its grid small rather than filling the GPU with idle blocks.
inline int coop_grid(int64_t want, int num_sms, int resident) {
  int64_t g = want < num_sms ? num_sms : want;
  if (g > resident) g = resident;
  if (g > kMaxGrid) g = kMaxGrid;
  return (int)g;
}

struct PerDeviceBlocks {
  std::mutex mu;
  int blocks[kMaxDevices] = {0};
  template <typename F>
  cudaError_t get(F setup, int* out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(mu);
    if (blocks[dev] == 0) {
      int b = 0;
      if ((e = setup(&b)) != cudaSuccess) return e;
      if (b < 1) return cudaErrorLaunchOutOfResources;
      blocks[dev] = b;
    }
    *out = blocks[dev];
    return cudaSuccess;
  }
};

// Each returns cudaGetLastError() of its launches.
cudaError_t launch_front(const Plan& p, cudaStream_t s);      // init, bounds, finalize, keys
cudaError_t launch_keys(const Plan& p, cudaStream_t s);
cudaError_t launch_radix(const Plan& p, cudaStream_t s);
cudaError_t launch_csort(const Plan& p, cudaStream_t s);
cudaError_t launch_rle(const Plan& p, cudaStream_t s);
cudaError_t launch_cell_prep(const Plan& p, cudaStream_t s);
cudaError_t launch_core(const Plan& p, cudaStream_t s);
cudaError_t launch_union(const Plan& p, cudaStream_t s);
cudaError_t launch_ids(const Plan& p, cudaStream_t s);
cudaError_t launch_labels(const Plan& p, cudaStream_t s);

}  // namespace dbs
