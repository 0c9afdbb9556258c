// dbs_capi.cu -- the C-ABI of include/dbscan_b200.h: workspace layout, the
// launch sequence of one pipeline run, profile / debug / batched / host-buffer
// forms.
//
// Reference functions replaced (ryanirl/dbscan-torch v0.2.0,
// csrc/cuda/dbscan_cuda.cu): dbscan2d_cuda_impl :531-750 (orchestration),
// dbscan2d_cuda :752-755, dbscan2d_cuda_profile :760-770 (same ten stage
// names, kStageNames :513-524), dbscan2d_cuda_debug :790-800 (same eleven
// intermediates, layout :777-789).
#include <cmath>
#include <cstring>
#include <mutex>

#include "../../include/dbscan_b200.h"
#include "dbs_internal.cuh"

static_assert(dbs::kNumTuned == DBS_NUM_TUNED && dbs::kTuneCount == DBS_TUNE_COUNT &&
                  dbs::kTuneCellPrep == DBS_TUNE_CELL_PREP && dbs::kTuneCore == DBS_TUNE_CORE &&
                  dbs::kTunePairs == DBS_TUNE_PAIRS && dbs::kTunePairScan == DBS_TUNE_PAIR_SCAN &&
                  dbs::kTuneLabels == DBS_TUNE_LABELS,
              "launch-shape indices of the C-ABI and the pipeline differ");

namespace dbs {
namespace {

constexpr size_t kAlign = 256;

inline size_t align_up(size_t v) { return (v + kAlign - 1) & ~(kAlign - 1); }

struct Carver {
  char* base;
  size_t off = 0;
  template <typename T>
  T* take(size_t count) {
    T* p = base ? reinterpret_cast<T*>(base + off) : nullptr;
    off = align_up(off + sizeof(T) * count);
    return p;
  }
};

// Lays out every array of one call. With base == nullptr only sizes.
size_t carve(int64_t n, int32_t nseg, char* base, Plan* p) {
  Plan q;
  std::memset(&q, 0, sizeof(q));
  Carver cv{base};
  const size_t N = (size_t)(n > 0 ? n : 1);
  const int32_t scan_tiles = (int32_t)((N + kScanTile - 1) / kScanTile);
  const int32_t ids_tiles = (int32_t)((N + kIdsTile - 1) / kIdsTile);
  q.desc = cv.take<Desc>(1);
  q.seg_off = cv.take<int64_t>((size_t)nseg + 1);
  q.seg_param = cv.take<SegParam>((size_t)nseg);
  q.seg_info = cv.take<SegInfo>((size_t)nseg);
  q.keys[0] = cv.take<uint64_t>(N);
  q.keys[1] = cv.take<uint64_t>(N);
  q.vals[0] = cv.take<uint32_t>(N);
  q.vals[1] = cv.take<uint32_t>(N);
  q.perm = cv.take<uint32_t>(N);
  q.xy = cv.take<float2>(N);
  q.is_core = cv.take<uint8_t>(N);
  q.chunk_count = cv.take<uint32_t>((size_t)kRadix * kMaxChunks);
  q.rle_status = cv.take<unsigned long long>((size_t)scan_tiles);
  q.ids_status = cv.take<unsigned long long>((size_t)ids_tiles);
  q.point_cell = cv.take<int32_t>(N);
  q.cell_start = cv.take<int32_t>(N + 1);
  q.cell_key = cv.take<uint64_t>(N);
  q.cell_seg = cv.take<int32_t>(N);
  q.bbox = cv.take<float4>(N);
  q.ngh = cv.take<int32_t>(N * kNgh);
  q.cell_status = cv.take<uint8_t>(N);
  q.uf = cv.take<int32_t>(N);
  q.root_rank = cv.take<int32_t>(N);
  q.cid = cv.take<int32_t>(N);
  q.qlist = cv.take<uint32_t>(N);
  q.blist = cv.take<uint32_t>(N);
  // Candidate pairs (c, nc > c) of one union pass: each unordered neighbour
  // pair is listed once, so at most 2 per cell in pass 0 (4 side
  // neighbours) and 10 in pass 1 (20 diagonal and outer neighbours).
  // Entries are counted in 32 bits: at most 2^32 - 1 (reached only beyond
  // 429M points; k_pairs reports an overflow in the status word).
  q.pair_cap = std::min<int64_t>(10 * (int64_t)N, 0xffffffffLL);
  q.plist = cv.take<int2>((size_t)q.pair_cap);
  q.dlist = cv.take<uint32_t>((size_t)q.pair_cap);
  q.dense_cap = kDenseFactor * (int64_t)N + kDenseSlack * (int64_t)nseg;
  q.cell_map = cv.take<int32_t>((size_t)q.dense_cap);
  q.big_cap = (int64_t)(N / kHugeCell) + 1;
  q.chunk_cap = (int64_t)(N / kHugeChunk) + q.big_cap + 1;
  q.big_cell = cv.take<int32_t>((size_t)q.big_cap);
  q.big_base = cv.take<unsigned long long>((size_t)q.big_cap);
  q.big_done = cv.take<uint32_t>((size_t)q.big_cap);
  q.big_chunk_box = cv.take<float4>((size_t)q.chunk_cap);
  q.bin_count = cv.take<uint32_t>((size_t)q.dense_cap);
  q.blk_sum = cv.take<uint32_t>((size_t)kMaxGrid);
  q.blk_ne = cv.take<uint32_t>((size_t)kMaxGrid);
  q.hot_key = cv.take<uint32_t>((size_t)kHotSlots);
  q.hot_cnt = cv.take<uint32_t>((size_t)kHotSlots);
  q.hot_cold = cv.take<uint32_t>((size_t)kHotSlots);
  q.hot_base = cv.take<uint32_t>((size_t)kHotSlots);
  q.n = n;
  q.nseg = nseg;
  q.scan_tiles = scan_tiles;
  q.ids_tiles = ids_tiles;
  for (int k = 0; k < kNumTuned; ++k) q.bps[k] = default_blocks_per_sm(k, n);
  if (p) *p = q;
  return cv.off;
}

// Radix-pass chunks: about three resident scatter blocks per SM, each
// owning a whole number of kSortTile tiles.
void set_chunking(Plan* p) {
  const int64_t tiles = (p->n + kSortTile - 1) / kSortTile;
  int64_t target = (int64_t)p->num_sms * 3;
  if (target > kMaxChunks) target = kMaxChunks;
  if (target < 1) target = 1;
  int64_t per = (tiles + target - 1) / target;
  if (per < 1) per = 1;
  p->chunk_tiles = (int32_t)per;
  p->sort_chunks = (int32_t)((tiles + per - 1) / per);
  if (p->sort_chunks < 1) p->sort_chunks = 1;
}

int num_sms_current() {
  static std::mutex mu;
  static int cache[64] = {0};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 148;
  std::lock_guard<std::mutex> lock(mu);
  if (dev >= 0 && dev < 64 && cache[dev] > 0) return cache[dev];
  int sms = 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0)
    sms = 148;
  if (dev >= 0 && dev < 64) cache[dev] = sms;
  return sms;
}

SegParam make_param(double eps, int64_t min_samples) {
  // dbscan_cuda.cu:547-550, computed on the host in IEEE float.
  SegParam sp;
  const float fl_eps = static_cast<float>(eps);
  sp.inv_r = std::sqrt(2.0f) / fl_eps;
  sp.eps_sq = fl_eps * fl_eps;
  sp.ms = static_cast<int32_t>(min_samples);
  sp.pad = 0;
  return sp;
}

int check_ws(const void* ws, size_t ws_bytes, size_t need) {
  if (ws == nullptr || (reinterpret_cast<uintptr_t>(ws) & (kAlign - 1)) != 0 || ws_bytes < need)
    return DBS_ERR_WORKSPACE;
  return DBS_OK;
}

int to_code(cudaError_t e) { return e == cudaSuccess ? DBS_OK : DBS_ERR_CUDA; }

// The launch sequence of one pipeline run. `evs` (nullable) receives the
// boundaries of the reference's ten stages.
int run_pipeline(const Plan& p, cudaStream_t s, cudaEvent_t* evs) {
  auto mark = [&](int i) -> cudaError_t {
    return evs ? cudaEventRecord(evs[i], s) : cudaSuccess;
  };
  cudaError_t e;
  if ((e = mark(0)) != cudaSuccess) return to_code(e);
  if ((e = launch_front(p, s)) != cudaSuccess) return to_code(e);            // cell_keys
  if ((e = mark(1)) != cudaSuccess) return to_code(e);
  if ((e = launch_csort(p, s)) != cudaSuccess) return to_code(e);            // sort_gather
  if ((e = launch_keys(p, s)) != cudaSuccess) return to_code(e);
  if ((e = launch_radix(p, s)) != cudaSuccess) return to_code(e);
  if ((e = mark(2)) != cudaSuccess) return to_code(e);
  if ((e = launch_rle(p, s)) != cudaSuccess) return to_code(e);              // boundary_scan
  if ((e = mark(3)) != cudaSuccess) return to_code(e);
  if ((e = launch_cell_prep(p, s)) != cudaSuccess) return to_code(e);        // build_ngh
  if ((e = mark(4)) != cudaSuccess) return to_code(e);
  if ((e = launch_core(p, s)) != cudaSuccess) return to_code(e);             // core_mark
  if ((e = mark(5)) != cudaSuccess) return to_code(e);
  if ((e = launch_union(p, s)) != cudaSuccess) return to_code(e);            // union_find
  if ((e = mark(6)) != cudaSuccess) return to_code(e);
  if ((e = launch_ids(p, s)) != cudaSuccess) return to_code(e);              // cluster_id
  if ((e = mark(7)) != cudaSuccess) return to_code(e);
  // core_labels, border_assign and unpermute are one kernel (k_labels); its
  // time is reported under border_assign.
  if ((e = mark(8)) != cudaSuccess) return to_code(e);
  if ((e = launch_labels(p, s)) != cudaSuccess) return to_code(e);           // border_assign
  if ((e = mark(9)) != cudaSuccess) return to_code(e);
  if ((e = mark(10)) != cudaSuccess) return to_code(e);
  return DBS_OK;
}

int prepare_single(const float* X, int64_t n, double eps, int64_t min_samples, int32_t* labels,
                   void* ws, size_t ws_bytes, Plan* p) {
  if (n < 0 || !(eps > 0.0) || min_samples < 1) return DBS_ERR_INVALID;
  if (n > (int64_t)INT32_MAX) return DBS_ERR_TOO_LARGE;
  if (n > 0 && (X == nullptr || labels == nullptr)) return DBS_ERR_INVALID;
  const size_t need = carve(n, 1, nullptr, nullptr);
  int rc = check_ws(ws, ws_bytes, need);
  if (rc != DBS_OK) return rc;
  carve(n, 1, static_cast<char*>(ws), p);
  p->X = reinterpret_cast<const float2*>(X);
  p->labels = labels;
  p->num_sms = num_sms_current();
  set_chunking(p);
  p->single = 1;
  p->single_param = make_param(eps, min_samples);
  return DBS_OK;
}

// ------------------------------------------------------------ debug export
// Writes the reference's intermediates in its own formats: the u64 packed
// key of every sorted point, the sorted coordinates, core labels before the
// border pass and final labels in sorted order, cluster id per cell.
__global__ void k_debug_export(Plan p, dbs_debug_buffers o) {
  const uint32_t lane = lane_id();
  const uint32_t C = p.desc->num_cells;
  while (true) {
    uint32_t c = 0;
    if (lane == 0) c = atomicAdd(&p.desc->ctr[kCtrDebug], 1u);
    c = __shfl_sync(0xffffffffu, c, 0);
    if (c >= C) break;
    const int32_t seg = p.cell_seg[c];
    const int32_t cid = p.cid[c];
    if (lane == 0 && o.cluster_id_per_cell) o.cluster_id_per_cell[c] = cid;
    const float inv_r = p.seg_param[seg].inv_r;
    for (int32_t i = p.cell_start[c] + lane; i < p.cell_start[c + 1]; i += 32) {
      const float2 v = p.xy[i];
      if (o.keys_sorted) {
        const uint32_t kx = (uint32_t)cell_coord(v.x, inv_r), ky = (uint32_t)cell_coord(v.y, inv_r);
        o.keys_sorted[i] = (int64_t)(((uint64_t)kx << 32) | ky);
      }
      if (o.xs) o.xs[i] = v.x;
      if (o.ys) o.ys[i] = v.y;
      const bool core = p.is_core[i] != 0;
      if (o.sorted_labels_pre_border) o.sorted_labels_pre_border[i] = core ? cid : -1;
      if (o.sorted_labels_final) o.sorted_labels_final[i] = p.labels[p.perm[i]];
    }
  }
}

int run_debug_export(const Plan& p, const dbs_debug_buffers& o, cudaStream_t s, int64_t n) {
  k_debug_export<<<p.num_sms * 8, 256, 0, s>>>(p, o);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return DBS_ERR_CUDA;
  if (o.perm && (e = cudaMemcpyAsync(o.perm, p.perm, sizeof(int32_t) * n, cudaMemcpyDeviceToDevice, s)) != cudaSuccess)
    return DBS_ERR_CUDA;
  if (o.is_core && (e = cudaMemcpyAsync(o.is_core, p.is_core, n, cudaMemcpyDeviceToDevice, s)) != cudaSuccess)
    return DBS_ERR_CUDA;
  return DBS_OK;
}

}  // namespace
}  // namespace dbs

using namespace dbs;

extern "C" {

size_t dbs_workspace_bytes(int64_t n_total, int32_t nseg) {
  if (n_total < 0 || nseg < 1) return 0;
  return carve(n_total, nseg, nullptr, nullptr);
}

int dbs_dbscan2d(const float* X, int64_t n, double eps, int64_t min_samples, int32_t* labels,
                 void* ws, size_t ws_bytes, void* stream) {
  Plan p;
  int rc = prepare_single(X, n, eps, min_samples, labels, ws, ws_bytes, &p);
  if (rc != DBS_OK || n == 0) return rc;
  return run_pipeline(p, static_cast<cudaStream_t>(stream), nullptr);
}

int dbs_dbscan2d_profile(const float* X, int64_t n, double eps, int64_t min_samples,
                         int32_t* labels, void* ws, size_t ws_bytes, void* stream,
                         float* stage_ms) {
  if (stage_ms == nullptr) return DBS_ERR_INVALID;
  for (int i = 0; i < DBS_NUM_STAGES; ++i) stage_ms[i] = 0.f;
  Plan p;
  int rc = prepare_single(X, n, eps, min_samples, labels, ws, ws_bytes, &p);
  if (rc != DBS_OK || n == 0) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  cudaEvent_t evs[DBS_NUM_STAGES + 1];
  int created = 0;
  for (; created <= DBS_NUM_STAGES; ++created)
    if (cudaEventCreate(&evs[created]) != cudaSuccess) break;
  if (created <= DBS_NUM_STAGES) {
    for (int i = 0; i < created; ++i) cudaEventDestroy(evs[i]);
    return DBS_ERR_CUDA;
  }
  rc = run_pipeline(p, s, evs);
  if (rc == DBS_OK && cudaStreamSynchronize(s) != cudaSuccess) rc = DBS_ERR_CUDA;
  if (rc == DBS_OK)
    for (int i = 0; i < DBS_NUM_STAGES; ++i)
      if (cudaEventElapsedTime(&stage_ms[i], evs[i], evs[i + 1]) != cudaSuccess) rc = DBS_ERR_CUDA;
  for (int i = 0; i <= DBS_NUM_STAGES; ++i) cudaEventDestroy(evs[i]);
  return rc;
}

int dbs_dbscan2d_debug(const float* X, int64_t n, double eps, int64_t min_samples,
                       int32_t* labels, void* ws, size_t ws_bytes, void* stream,
                       const dbs_debug_buffers* out, int64_t* num_cells) {
  return dbs_dbscan2d_debug_ex(X, n, eps, min_samples, labels, ws, ws_bytes, stream, out, num_cells,
                               DBS_DEBUG_STABLE_SORT);
}

int dbs_dbscan2d_debug_ex(const float* X, int64_t n, double eps, int64_t min_samples,
                          int32_t* labels, void* ws, size_t ws_bytes, void* stream,
                          const dbs_debug_buffers* out, int64_t* num_cells, int32_t flags) {
  if (out == nullptr || num_cells == nullptr || (flags & ~DBS_DEBUG_STABLE_SORT) != 0)
    return DBS_ERR_INVALID;
  *num_cells = 0;
  Plan p;
  int rc = prepare_single(X, n, eps, min_samples, labels, ws, ws_bytes, &p);
  if (rc != DBS_OK || n == 0) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // Stable sort: perm and sorted coordinates as the reference's.
  p.force_radix = (flags & DBS_DEBUG_STABLE_SORT) ? 1 : 0;
  rc = run_pipeline(p, s, nullptr);
  if (rc != DBS_OK) return rc;
  rc = run_debug_export(p, *out, s, n);
  if (rc != DBS_OK) return rc;
  uint32_t C = 0;
  if (cudaMemcpyAsync(&C, &p.desc->num_cells, sizeof(C), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return DBS_ERR_CUDA;
  *num_cells = C;
  if (out->cell_start &&
      cudaMemcpyAsync(out->cell_start, p.cell_start, sizeof(int32_t) * ((size_t)C + 1),
                      cudaMemcpyDeviceToDevice, s) != cudaSuccess)
    return DBS_ERR_CUDA;
  if (out->uf && cudaMemcpyAsync(out->uf, p.uf, sizeof(int32_t) * (size_t)C, cudaMemcpyDeviceToDevice,
                                 s) != cudaSuccess)
    return DBS_ERR_CUDA;
  return cudaStreamSynchronize(s) == cudaSuccess ? DBS_OK : DBS_ERR_CUDA;
}

int dbs_fill_seg_params(const double* eps, const int64_t* min_samples, int32_t nseg,
                        void* params_host) {
  if (nseg < 1 || eps == nullptr || min_samples == nullptr || params_host == nullptr)
    return DBS_ERR_INVALID;
  SegParam* out = static_cast<SegParam*>(params_host);
  for (int32_t s = 0; s < nseg; ++s) {
    if (!(eps[s] > 0.0) || min_samples[s] < 1) return DBS_ERR_INVALID;
    out[s] = make_param(eps[s], min_samples[s]);
  }
  return DBS_OK;
}

int dbs_default_launch_shape(int64_t n_total, dbs_launch_shape* out) {
  if (out == nullptr || n_total < 0) return DBS_ERR_INVALID;
  for (int k = 0; k < kNumTuned; ++k) out->blocks_per_sm[k] = default_blocks_per_sm(k, n_total);
  return DBS_OK;
}

int dbs_dbscan2d_batched_device(const float* X, int64_t n_total, int32_t nseg,
                                const int64_t* seg_offsets_dev, const void* seg_params_dev,
                                int32_t* labels, void* ws, size_t ws_bytes, void* stream) {
  return dbs_dbscan2d_batched_device_shaped(X, n_total, nseg, seg_offsets_dev, seg_params_dev, labels,
                                            ws, ws_bytes, nullptr, stream);
}

int dbs_dbscan2d_batched_device_shaped(const float* X, int64_t n_total, int32_t nseg,
                                       const int64_t* seg_offsets_dev, const void* seg_params_dev,
                                       int32_t* labels, void* ws, size_t ws_bytes,
                                       const dbs_launch_shape* shape, void* stream) {
  if (shape != nullptr)
    for (int k = 0; k < kNumTuned; ++k)
      if (shape->blocks_per_sm[k] < 0 || shape->blocks_per_sm[k] > DBS_SHAPE_MAX_BLOCKS_PER_SM)
        return DBS_ERR_INVALID;
  if (n_total < 0 || nseg < 1 || seg_offsets_dev == nullptr || seg_params_dev == nullptr)
    return DBS_ERR_INVALID;
  if (n_total > (int64_t)INT32_MAX) return DBS_ERR_TOO_LARGE;
  if (n_total > 0 && (X == nullptr || labels == nullptr)) return DBS_ERR_INVALID;
  const size_t need = carve(n_total, nseg, nullptr, nullptr);
  int rc = check_ws(ws, ws_bytes, need);
  if (rc != DBS_OK) return rc;
  if (n_total == 0) return DBS_OK;
  Plan p;
  carve(n_total, nseg, static_cast<char*>(ws), &p);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (cudaMemcpyAsync(p.seg_off, seg_offsets_dev, sizeof(int64_t) * ((size_t)nseg + 1),
                      cudaMemcpyDeviceToDevice, s) != cudaSuccess ||
      cudaMemcpyAsync(p.seg_param, seg_params_dev, sizeof(SegParam) * (size_t)nseg,
                      cudaMemcpyDeviceToDevice, s) != cudaSuccess)
    return DBS_ERR_CUDA;
  p.X = reinterpret_cast<const float2*>(X);
  p.labels = labels;
  p.num_sms = num_sms_current();
  if (shape != nullptr)
    for (int k = 0; k < kNumTuned; ++k)
      if (shape->blocks_per_sm[k] > 0) p.bps[k] = shape->blocks_per_sm[k];
  set_chunking(&p);
  p.single = 0;
  return run_pipeline(p, s, nullptr);
}

int dbs_dbscan2d_batched(const float* X, const int64_t* seg_offsets, const double* eps,
                         const int64_t* min_samples, int32_t nseg, int32_t* labels, void* ws,
                         size_t ws_bytes, void* stream) {
  if (nseg < 1 || seg_offsets == nullptr || eps == nullptr || min_samples == nullptr)
    return DBS_ERR_INVALID;
  if (seg_offsets[0] != 0) return DBS_ERR_INVALID;
  for (int32_t s = 0; s < nseg; ++s)
    if (seg_offsets[s + 1] < seg_offsets[s] || !(eps[s] > 0.0) || min_samples[s] < 1)
      return DBS_ERR_INVALID;
  const int64_t n_total = seg_offsets[nseg];
  if (n_total > (int64_t)INT32_MAX) return DBS_ERR_TOO_LARGE;
  if (n_total > 0 && (X == nullptr || labels == nullptr)) return DBS_ERR_INVALID;
  const size_t need = carve(n_total, nseg, nullptr, nullptr);
  int rc = check_ws(ws, ws_bytes, need);
  if (rc != DBS_OK) return rc;
  if (n_total == 0) return DBS_OK;
  Plan p;
  carve(n_total, nseg, static_cast<char*>(ws), &p);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // Pageable host sources: cudaMemcpyAsync returns once the host bytes are
  // staged, so the temporary table may be freed right after the call.
  SegParam* params = new SegParam[(size_t)nseg];
  dbs_fill_seg_params(eps, min_samples, nseg, params);
  cudaError_t e1 = cudaMemcpyAsync(p.seg_off, seg_offsets, sizeof(int64_t) * ((size_t)nseg + 1),
                                   cudaMemcpyHostToDevice, s);
  cudaError_t e2 = cudaMemcpyAsync(p.seg_param, params, sizeof(SegParam) * (size_t)nseg,
                                   cudaMemcpyHostToDevice, s);
  delete[] params;
  if (e1 != cudaSuccess || e2 != cudaSuccess) return DBS_ERR_CUDA;
  p.X = reinterpret_cast<const float2*>(X);
  p.labels = labels;
  p.num_sms = num_sms_current();
  set_chunking(&p);
  p.single = 0;
  return run_pipeline(p, s, nullptr);
}

size_t dbs_host_workspace_bytes(int64_t n) {
  if (n < 0) return 0;
  const size_t N = (size_t)(n > 0 ? n : 1);
  return carve(n, 1, nullptr, nullptr) + align_up(sizeof(float2) * N) + align_up(sizeof(int32_t) * N);
}

int dbs_dbscan2d_host(const float* X_host, int64_t n, double eps, int64_t min_samples,
                      int32_t* labels_host, void* ws, size_t ws_bytes, void* stream) {
  if (n < 0 || !(eps > 0.0) || min_samples < 1) return DBS_ERR_INVALID;
  if (n > (int64_t)INT32_MAX) return DBS_ERR_TOO_LARGE;
  if (n == 0) return DBS_OK;
  if (X_host == nullptr || labels_host == nullptr) return DBS_ERR_INVALID;
  const size_t need = dbs_host_workspace_bytes(n);
  int rc = check_ws(ws, ws_bytes, need);
  if (rc != DBS_OK) return rc;
  const size_t core = carve(n, 1, nullptr, nullptr);
  char* base = static_cast<char*>(ws);
  float* Xd = reinterpret_cast<float*>(base + core);
  int32_t* Ld = reinterpret_cast<int32_t*>(base + core + align_up(sizeof(float2) * (size_t)n));
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (cudaMemcpyAsync(Xd, X_host, sizeof(float2) * (size_t)n, cudaMemcpyHostToDevice, s) != cudaSuccess)
    return DBS_ERR_CUDA;
  rc = dbs_dbscan2d(Xd, n, eps, min_samples, Ld, ws, core, stream);
  if (rc != DBS_OK) return rc;
  if (cudaMemcpyAsync(labels_host, Ld, sizeof(int32_t) * (size_t)n, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return DBS_ERR_CUDA;
  uint32_t st = 0;
  rc = dbs_read_status(ws, stream, &st);
  if (rc != DBS_OK) return rc;
  return st ? DBS_ERR_DEVICE : DBS_OK;
}

int dbs_read_status(const void* ws, void* stream, uint32_t* status) {
  if (ws == nullptr || status == nullptr) return DBS_ERR_INVALID;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const Desc* d = static_cast<const Desc*>(ws);
  if (cudaMemcpyAsync(status, &d->status, sizeof(uint32_t), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return DBS_ERR_CUDA;
  return DBS_OK;
}

int dbs_read_plan(const void* ws, void* stream, int64_t* num_cells, int32_t* key_bits,
                  int32_t* passes, int32_t* key_bytes) {
  if (ws == nullptr) return DBS_ERR_INVALID;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const Desc* d = static_cast<const Desc*>(ws);
  Desc h;
  if (cudaMemcpyAsync(&h, d, sizeof(Desc), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return DBS_ERR_CUDA;
  if (num_cells) *num_cells = h.num_cells;
  if (key_bits) *key_bits = (int32_t)h.nbits;
  if (passes) *passes = h.dense_sort ? 0 : (int32_t)h.npasses;
  if (key_bytes) *key_bytes = h.key64 ? 8 : 4;
  return DBS_OK;
}

int dbs_read_stats(const void* ws, void* stream, dbs_run_stats* out) {
  if (ws == nullptr || out == nullptr) return DBS_ERR_INVALID;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  Desc h;
  if (cudaMemcpyAsync(&h, ws, sizeof(Desc), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return DBS_ERR_CUDA;
  out->num_cells = h.num_cells;
  out->key_bits = (int32_t)h.nbits;
  out->passes = h.dense_sort ? 0 : (int32_t)h.npasses;
  out->key_bytes = h.key64 ? 8 : 4;
  out->hot_slots = (int32_t)h.hot_used;
  out->sort_form = (int32_t)h.dense_sort;
  out->queries = h.q_count;
  out->border = h.b_count;
  // The flatten between the passes saved pass 0's counts; pass 1's are the
  // live counters.
  out->pairs[0] = h.ring_pairs[0];
  out->pairs[1] = h.p_count;
  out->warp_pairs[0] = h.ring_warp[0];
  out->warp_pairs[1] = h.d_count;
  return DBS_OK;
}

const char* dbs_strerror(int code) {
  switch (code) {
    case DBS_OK: return "ok";
    case DBS_ERR_INVALID: return "invalid argument";
    case DBS_ERR_WORKSPACE: return "workspace missing, misaligned or too small";
    case DBS_ERR_TOO_LARGE: return "too many points (n must be < 2^31)";
    case DBS_ERR_CUDA: return "CUDA runtime error";
    case DBS_ERR_DEVICE: return "device-side failure (bounded wait exceeded)";
    case DBS_ERR_STATIC_LIMIT:
      return "too many points for the built-in scratch (n must be <= DBS_STATIC_MAX_POINTS = 16384); "
             "use dbs_dbscan2d with a workspace";
    default: return "unknown error";
  }
}

const char* dbs_stage_name(int stage) {
  // Stage names of the reference (dbscan_cuda.cu:513-524).
  static const char* const kNames[DBS_NUM_STAGES] = {
      "cell_keys", "sort_gather", "boundary_scan", "build_ngh", "core_mark",
      "union_find", "cluster_id", "core_labels", "border_assign", "unpermute"};
  if (stage < 0 || stage >= DBS_NUM_STAGES) return nullptr;
  return kNames[stage];
}

}  // extern "C"

// ------------------------------------------------------ built-in scratch form
// dbs_dbscan2d_static: the pipeline of dbs_dbscan2d on a workspace carved
// out of a fixed array in this library's device image. Some callers have no
// means to allocate device memory when they cluster -- a host plugin handed
// device pointers but no allocator, an out-of-memory handler, a loop that
// cannot afford the device-wide synchronisation of cudaMalloc / cudaFree --
// so this form calls no allocating routine at all: the array is part of the
// module image, its address is looked up once per device, and the launch
// sequence is the one every other entry point runs.

// The first kernel of every call (k_init) resets every counter, flag and
// look-back word the later kernels read, so no byte has to start at zero.
static __device__ __align__(256) unsigned char g_dbs_static_scratch[DBS_STATIC_SCRATCH_BYTES];

namespace dbs {
namespace {

constexpr int kStaticDevices = 64;
std::mutex g_static_mu;
void* g_static_addr[kStaticDevices] = {nullptr};

// Address of g_dbs_static_scratch on the current device. Set-up happens on
// the first call made with that device current.
int static_scratch(void** out) {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kStaticDevices) return DBS_ERR_CUDA;
  std::lock_guard<std::mutex> lock(g_static_mu);
  if (g_static_addr[dev] == nullptr) {
    void* a = nullptr;
    if (cudaGetSymbolAddress(&a, g_dbs_static_scratch) != cudaSuccess || a == nullptr)
      return DBS_ERR_CUDA;
    g_static_addr[dev] = a;
  }
  *out = g_static_addr[dev];
  return DBS_OK;
}

}  // namespace
}  // namespace dbs

extern "C" int dbs_dbscan2d_static(const float* X, int64_t n, double eps, int64_t min_samples,
                                   int32_t* labels, uint32_t* status, void* stream) {
  if (n < 0 || !(eps > 0.0) || min_samples < 1) return DBS_ERR_INVALID;
  if (n > DBS_STATIC_MAX_POINTS) return DBS_ERR_STATIC_LIMIT;
  if (n > 0 && (X == nullptr || labels == nullptr)) return DBS_ERR_INVALID;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (n == 0) {
    if (status && cudaMemsetAsync(status, 0, sizeof(uint32_t), s) != cudaSuccess) return DBS_ERR_CUDA;
    return DBS_OK;
  }
  void* ws = nullptr;
  int rc = static_scratch(&ws);
  if (rc != DBS_OK) return rc;
  Plan p;
  rc = prepare_single(X, n, eps, min_samples, labels, ws, DBS_STATIC_SCRATCH_BYTES, &p);
  if (rc != DBS_OK) return rc;
  rc = run_pipeline(p, s, nullptr);
  if (rc != DBS_OK) return rc;
  if (status && cudaMemcpyAsync(status, &p.desc->status, sizeof(uint32_t), cudaMemcpyDeviceToDevice,
                                s) != cudaSuccess)
    return DBS_ERR_CUDA;
  return DBS_OK;
}
