/*
 * dbscan_b200.h -- C-ABI of the sm_100a grid-hashed 2D DBSCAN library
 * (libdbscan_b200.so).
 *
 * Drop-in boundary for the GPU path of ryanirl/dbscan-torch v0.2.0. Each
 * entry point below replaces one function of the reference's CUDA translation
 * unit (csrc/cuda/dbscan_cuda.cu) that its pybind module binds through
 * csrc/extension.cpp; the torch extension of this repository (_C) is a thin
 * C++ layer that validates tensors exactly like extension.cpp:26-31 and calls
 * these functions. No torch, thrust or CUB types cross this boundary: plain
 * pointers, sizes and a cudaStream_t passed as void*.
 *
 * Conventions
 *   - X is float32 (n, 2) row-major (AoS x, y), device memory unless noted.
 *   - labels are int32 (n,), -1 = noise, else a cluster id in [0, k) numbered
 *     exactly like the reference CUDA path (rank of each cluster's smallest
 *     cell in ascending unsigned cell-key order).
 *   - eps and min_samples follow dbscan_cuda.cu:547-550: fl_eps = (float)eps,
 *     inv_r = sqrtf(2)/fl_eps, eps_sq = fl_eps*fl_eps, ms = (int32)min_samples.
 *   - ws is a caller-owned device workspace of at least
 *     dbs_workspace_bytes(n, nseg) bytes, 256-byte aligned. The library never
 *     allocates device memory; calls on one workspace must not overlap.
 *   - All work is enqueued on `stream` (a cudaStream_t; NULL = legacy default
 *     stream). Unless stated otherwise an entry point does not synchronise:
 *     the enqueue sequence holds no host read-back, so it can be captured in
 *     a CUDA graph. Device-side failures (a bounded wait that ran out) are
 *     recorded in the workspace and read with dbs_read_status().
 *   - Return value: DBS_OK or a DBS_ERR_* code (see dbs_strerror()).
 */
#ifndef DBSCAN_B200_H_
#define DBSCAN_B200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DBS_OK 0
#define DBS_ERR_INVALID 1       /* bad argument: shape, eps <= 0, min_samples < 1, n < 0 */
#define DBS_ERR_WORKSPACE 2     /* ws NULL, misaligned or smaller than required */
#define DBS_ERR_TOO_LARGE 3     /* n >= 2^31 (the reference indexes points with int32) */
#define DBS_ERR_CUDA 4          /* a CUDA runtime call failed */
#define DBS_ERR_DEVICE 5        /* device status word non-zero (see dbs_read_status) */

/* Device status bits (dbs_read_status). */
#define DBS_STATUS_LOOKBACK 1u  /* a decoupled look-back wait reached its cap */
#define DBS_STATUS_FIND 2u      /* a union-find walk reached its cap */
#define DBS_STATUS_KEYSPACE 4u  /* batched cell-key ranges overflowed 64 bits */
#define DBS_STATUS_BARRIER 8u   /* a grid-wide barrier wait reached its cap */
#define DBS_STATUS_CAPACITY 16u /* a work list (union-find cell pairs, at most 2^32 - 1)
                                   received more entries than it holds, or a sorted
                                   position fell outside [0, n) (internal check of
                                   range only: two points sharing one position, or a
                                   position left unfilled, would not set it) */

#define DBS_NUM_STAGES 10

/* Bytes of device workspace for nseg clouds holding n_total points. */
size_t dbs_workspace_bytes(int64_t n_total, int32_t nseg);

/* Plain call. Replaces dbscan2d_cuda (dbscan_cuda.cu:752-755), bound as
 * _C.dbscan2d (extension.cpp:33-45, 67-70). n == 0 is a no-op. */
int dbs_dbscan2d(const float* X, int64_t n, double eps, int64_t min_samples,
                 int32_t* labels, void* ws, size_t ws_bytes, void* stream);

/* Profile call. Replaces dbscan2d_cuda_profile (dbscan_cuda.cu:760-770),
 * bound as _C.dbscan2d_profile (extension.cpp:52-63, 71-74). Fills
 * stage_ms[DBS_NUM_STAGES] with the GPU time of each of the reference's ten
 * stages (names from dbs_stage_name()). Synchronises the stream. */
int dbs_dbscan2d_profile(const float* X, int64_t n, double eps, int64_t min_samples,
                         int32_t* labels, void* ws, size_t ws_bytes, void* stream,
                         float* stage_ms);

/* Debug call. Replaces dbscan2d_cuda_debug (dbscan_cuda.cu:790-800), bound as
 * _C.dbscan2d_cuda_debug (extension.cpp:76-79). Writes the reference's
 * per-stage intermediates (layout dbscan_cuda.cu:777-789) into caller device
 * buffers; cell-sized buffers need capacity n (cell_start n + 1). Any pointer
 * may be NULL. Synchronises the stream and returns num_cells in *num_cells. */
typedef struct dbs_debug_buffers {
  int64_t* keys_sorted;          /* (n) u64-packed (u32)kx << 32 | (u32)ky, sorted */
  int32_t* perm;                 /* (n) sorted position -> input index */
  float* xs;                     /* (n) sorted x */
  float* ys;                     /* (n) sorted y */
  uint8_t* is_core;              /* (n) sorted order */
  int32_t* cell_start;           /* (num_cells + 1) */
  int32_t* cluster_id_per_cell;  /* (num_cells) */
  int32_t* uf;                   /* (num_cells) flattened roots */
  int32_t* sorted_labels_pre_border; /* (n) core labels in sorted order */
  int32_t* sorted_labels_final;  /* (n) final labels in sorted order */
} dbs_debug_buffers;

int dbs_dbscan2d_debug(const float* X, int64_t n, double eps, int64_t min_samples,
                       int32_t* labels, void* ws, size_t ws_bytes, void* stream,
                       const dbs_debug_buffers* out, int64_t* num_cells);

/* Batched call (no counterpart in the reference; the reference handles one
 * cloud per dbscan2d call). nseg clouds are concatenated in X; cloud s owns
 * rows [seg_offsets[s], seg_offsets[s+1]) and has its own eps[s] and
 * min_samples[s]. seg_offsets, eps and min_samples are HOST arrays; labels
 * of cloud s land in the same rows of `labels`, each cloud numbered from 0
 * exactly as a plain call on that cloud alone. One pipeline launch sequence
 * covers every cloud. */
int dbs_dbscan2d_batched(const float* X, const int64_t* seg_offsets, const double* eps,
                         const int64_t* min_samples, int32_t nseg, int32_t* labels,
                         void* ws, size_t ws_bytes, void* stream);

/* Batched call with the per-cloud table already on the device, for CUDA
 * graph capture. seg_offsets_dev: int64 (nseg + 1); seg_params_dev: nseg
 * records of {float inv_r, float eps_sq, int32 ms, int32 pad} computed as in
 * the conventions above (dbs_fill_seg_params fills such a table on the host). */
int dbs_dbscan2d_batched_device(const float* X, int64_t n_total, int32_t nseg,
                                const int64_t* seg_offsets_dev, const void* seg_params_dev,
                                int32_t* labels, void* ws, size_t ws_bytes, void* stream);

/* Launch shape (no counterpart in the reference, whose kernels take fixed
 * grids sized by the work). blocks_per_sm[k] is the grid of tuned kernel k
 * in blocks per SM; 0 keeps the built-in value (dbs_default_launch_shape).
 * The tuned kernels all walk their work with grid-stride loops or dynamic
 * work counters, so labels do not depend on the shape, only the time does.
 * Valid entries: 0 .. DBS_SHAPE_MAX_BLOCKS_PER_SM. */
#define DBS_NUM_TUNED 6
#define DBS_TUNE_COUNT 0      /* per-key point counts of the counting sort */
#define DBS_TUNE_CELL_PREP 1  /* cell boxes, neighbour rows, point classes */
#define DBS_TUNE_CORE 2       /* core counts of the query points */
#define DBS_TUNE_PAIRS 3      /* candidate cell pairs (both rings) */
#define DBS_TUNE_PAIR_SCAN 4  /* pair tests and unions (both rings) */
#define DBS_TUNE_LABELS 5     /* border assignment, core labels, unpermute */
#define DBS_SHAPE_MAX_BLOCKS_PER_SM 32

typedef struct dbs_launch_shape {
  int32_t blocks_per_sm[DBS_NUM_TUNED];
} dbs_launch_shape;

/* The built-in shape of a run over n_total points (every entry non-zero):
 * the per-key count 6 blocks per SM (the blocks resident at once), the label
 * pass 32 up to 2^24 points and 8 above, every other kernel 8. */
int dbs_default_launch_shape(int64_t n_total, dbs_launch_shape* out);

/* dbs_dbscan2d_batched_device with a launch shape (NULL = built-in). An entry
 * outside 0 .. DBS_SHAPE_MAX_BLOCKS_PER_SM returns DBS_ERR_INVALID before any
 * CUDA call. */
int dbs_dbscan2d_batched_device_shaped(const float* X, int64_t n_total, int32_t nseg,
                                       const int64_t* seg_offsets_dev, const void* seg_params_dev,
                                       int32_t* labels, void* ws, size_t ws_bytes,
                                       const dbs_launch_shape* shape, void* stream);

/* Host helper: fills nseg 16-byte parameter records (see above). */
int dbs_fill_seg_params(const double* eps, const int64_t* min_samples, int32_t nseg,
                        void* params_host);

/* Host-buffer call: X and labels in HOST memory (pinned for asynchronous
 * copies). Copies in, runs the plain pipeline, copies out and synchronises.
 * ws must hold dbs_host_workspace_bytes(n). This is the end-to-end form of
 * _C.dbscan2d for a CPU tensor. */
size_t dbs_host_workspace_bytes(int64_t n);
int dbs_dbscan2d_host(const float* X_host, int64_t n, double eps, int64_t min_samples,
                      int32_t* labels_host, void* ws, size_t ws_bytes, void* stream);

/* Synchronises the stream and returns the device status word of the last
 * call on this workspace (0 = no failure; DBS_STATUS_* bits otherwise). */
int dbs_read_status(const void* ws, void* stream, uint32_t* status);

/* Shape of the last call on this workspace, read after synchronising the
 * stream: number of cells (distinct occupied grid cells over all clouds),
 * significant bits of the compacted cell keys, radix passes that ran (0 when
 * every cloud fit the dense key space and the counting sort ran instead), and
 * bytes per stored key (4 or 8). Any output pointer may be NULL. */
int dbs_read_plan(const void* ws, void* stream, int64_t* num_cells, int32_t* key_bits,
                  int32_t* passes, int32_t* key_bytes);

/* Work counts of the last call on this workspace, read after synchronising
 * the stream (no counterpart in the reference, which keeps no counters; the
 * figures size the work of each stage for profiling and tests):
 *   num_cells, key_bits, passes, key_bytes  as dbs_read_plan
 *   hot_slots    occupied slots of the counting sort's 64-slot hot-key table
 *                (keys that >= 8 lanes of one 32-point row share)
 *   queries      points of cells below min_samples (counted by distance tests)
 *   border       non-core points (border assignment candidates)
 *   pairs[r]     candidate core-cell pairs listed by union pass r (0: side
 *                neighbours, 1: diagonal and outer ring)
 *   warp_pairs[r] of those, pairs scanned warp-cooperatively (over budget)
 *   sort_form    0 radix sort (sparse key space, or the debug entry's stable
 *                sort), 1 counting sort over the dense key space */
typedef struct dbs_run_stats {
  int64_t num_cells;
  int32_t key_bits;
  int32_t passes;
  int32_t key_bytes;
  int32_t hot_slots;
  int32_t sort_form;
  int64_t queries;
  int64_t border;
  int64_t pairs[2];
  int64_t warp_pairs[2];
} dbs_run_stats;

int dbs_read_stats(const void* ws, void* stream, dbs_run_stats* out);

/* Debug call with a choice of sort (no counterpart in the reference).
 * flags = 0: the sort of the plain call -- the counting sort over a dense key
 * space, which places the points of one cell in arrival order, so perm,
 * xs, ys, is_core and the sorted labels are permuted within each cell
 * relative to the reference while keys_sorted, cell_start,
 * cluster_id_per_cell, uf and every label are the reference's.
 * flags = DBS_DEBUG_STABLE_SORT: as dbs_dbscan2d_debug (stable radix sort,
 * every intermediate in the reference's order). */
#define DBS_DEBUG_STABLE_SORT 1
int dbs_dbscan2d_debug_ex(const float* X, int64_t n, double eps, int64_t min_samples,
                          int32_t* labels, void* ws, size_t ws_bytes, void* stream,
                          const dbs_debug_buffers* out, int64_t* num_cells, int32_t flags);

const char* dbs_strerror(int code);
const char* dbs_stage_name(int stage);

/* ---------------------------------------------------------------------------
 * Built-in scratch form. No counterpart in the reference: its extension
 * always allocates through torch.
 *
 * dbs_dbscan2d_static runs the same pipeline as dbs_dbscan2d and returns the
 * same labels, but takes no workspace and allocates nothing: its scratch is a
 * fixed array of DBS_STATIC_SCRATCH_BYTES inside the library's device image,
 * enough for clouds of up to DBS_STATIC_MAX_POINTS points. It serves callers
 * that cannot allocate device memory when they cluster: a host plugin that is
 * handed device pointers but no allocator, code running inside an
 * out-of-memory handler or with the device memory already used up, and
 * latency-bound loops that must not take the device-wide synchronisation of
 * cudaMalloc / cudaFree.
 *
 *   - n > DBS_STATIC_MAX_POINTS is rejected with DBS_ERR_STATIC_LIMIT before
 *     any CUDA call; use dbs_dbscan2d with a workspace for larger clouds.
 *   - The first call made with a device current does the set-up for that
 *     device: it looks up the address of the scratch array there
 *     (cudaGetSymbolAddress, which may load the library's device code onto
 *     the device). Make that first call before any stream capture begins.
 *     The address is kept for the life of the process; after a
 *     cudaDeviceReset of that device this entry point must not be used.
 *   - Nothing in the scratch has to start at zero: the first kernel of every
 *     call resets each counter, flag and look-back word the later kernels
 *     read.
 *   - All calls on one device share the one array. Calls whose work overlaps
 *     on the device race on it and return wrong labels: issue them on one
 *     stream, or order them (events, synchronisation) across streams and
 *     host threads. Calls on different devices do not interact.
 *   - status (nullable, device memory) receives the call's device status
 *     word (0, or DBS_STATUS_* bits) by a stream-ordered copy.
 *   - n == 0 is a no-op (a non-NULL status is set to 0).
 */
#define DBS_STATIC_MAX_POINTS 16384
#define DBS_STATIC_SCRATCH_BYTES (8u << 20)
#define DBS_ERR_STATIC_LIMIT 6  /* n > DBS_STATIC_MAX_POINTS (dbs_dbscan2d_static) */

int dbs_dbscan2d_static(const float* X, int64_t n, double eps, int64_t min_samples,
                        int32_t* labels, uint32_t* status, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* DBSCAN_B200_H_ */
