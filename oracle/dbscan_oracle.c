/*
 * dbscan_oracle.c -- CPU restatement of the reference CUDA DBSCAN path.
 *
 * TEST INFRASTRUCTURE ONLY: this file is the checker. Only tests/, the smoke
 * check and the bench's CPU-baseline leg may load it; the product path never
 * does.
 *
 * It restates, stage for stage and in plain C, the label semantics of
 * csrc/cuda/dbscan_cuda.cu of ryanirl/dbscan-torch v0.2.0 (the reference's GPU
 * path, whose labels the product must match bit for bit):
 *
 *   stage 1  cell keys          dbscan_cuda.cu:47-66   (pack_key, k_cell_keys)
 *   stage 2  stable u64 sort    dbscan_cuda.cu:582-594 (sort_by_key, k_gather_xy)
 *   stage 3  run-length cells   dbscan_cuda.cu:84-120  (boundary flags, scan)
 *            cell bounding box  dbscan_cuda.cu:162-177 (k_cell_bbox)
 *   stage 4  5x5 neighbour tbl  dbscan_cuda.cu:125-150 (binsearch_cell, k_build_ngh)
 *   stage 5  core marking       dbscan_cuda.cu:183-263 (pass1, pass2, cell_status)
 *   stage 6  cell union-find    dbscan_cuda.cu:277-378 (k_unite_pairs, flatten)
 *   stage 7  cluster ids        dbscan_cuda.cu:383-404 (root flag, exclusive scan)
 *   stage 8  core labels        dbscan_cuda.cu:409-417
 *   stage 9  border assignment  dbscan_cuda.cu:427-470 (argmin of (d2, perm[j]))
 *   stage 10 unpermute          dbscan_cuda.cu:475-481
 *
 * Floating point follows the reference build (setup.py:77-83 compiles device
 * code with --use_fast_math): every single-precision operation flushes
 * subnormal inputs and results to zero, and the squared distance
 * `ex*ex + ey*ey` may be contracted into one fused multiply-add. Which operand
 * the compiler fuses is not visible in the source, so each of the seven call
 * sites takes a form parameter (unfused, fma(ex,ex,ey*ey), fma(ey,ey,ex*ex));
 * the forms the reference build actually uses were settled by feeding it
 * inputs on which the forms disagree and comparing labels.
 *
 * Host-side scalars follow dbscan_cuda.cu:547-549: fl_eps = (float)eps,
 * inv_r = sqrtf(2)/fl_eps and eps_sq = fl_eps*fl_eps in IEEE float (no flush).
 *
 * Build: see oracle/Makefile (gcc -O2 -ffp-contract=off, no fast-math).
 */
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORACLE_NOISE (-1)

enum { FORM_UNFUSED = 0, FORM_FMA_X = 1, FORM_FMA_Y = 2 };

/* Call sites whose arithmetic form is a parameter. */
enum {
  SITE_CORE_BOX = 0,   /* point_box_d2 in k_core_pass2        :235 */
  SITE_CORE_PAIR = 1,  /* ex*ex+ey*ey in k_core_pass2         :239 */
  SITE_UNITE_BB = 2,   /* box_box_d2 in k_unite_pairs         :351 */
  SITE_UNITE_BOX = 3,  /* point_box_d2 in k_unite_pairs       :359 */
  SITE_UNITE_PAIR = 4, /* ex*ex+ey*ey in k_unite_pairs        :363 */
  SITE_BORDER_BOX = 5, /* point_box_d2 in k_border_assign     :453 */
  SITE_BORDER_PAIR = 6,/* ex*ex+ey*ey in k_border_assign      :458 */
  NUM_SITES = 7
};

/* ---------------------------------------------------------------- float ops */
static inline float fz(float v) { return (fabsf(v) < FLT_MIN) ? copysignf(0.0f, v) : v; }
static inline float fmul(float a, float b) { return fz(fz(a) * fz(b)); }
static inline float fsub(float a, float b) { return fz(fz(a) - fz(b)); }
static inline float fadd(float a, float b) { return fz(fz(a) + fz(b)); }
static inline float ffma(float a, float b, float c) { return fz(fmaf(fz(a), fz(b), fz(c))); }
static inline float fmaxz(float a, float b) { return fmaxf(fz(a), fz(b)); }
static inline float fminz(float a, float b) { return fminf(fz(a), fz(b)); }
static inline int fle(float a, float b) { return fz(a) <= fz(b); }
static inline int flt(float a, float b) { return fz(a) < fz(b); }
static inline int feq(float a, float b) { return fz(a) == fz(b); }

/* ex*ex + ey*ey in the given form. */
static inline float sq2(float ex, float ey, int form) {
  switch (form) {
    case FORM_FMA_X: return ffma(ex, ex, fmul(ey, ey));
    case FORM_FMA_Y: return ffma(ey, ey, fmul(ex, ex));
    default: return fadd(fmul(ex, ex), fmul(ey, ey));
  }
}

/* dbscan_cuda.cu:183-187 */
static inline float point_box_d2(float x, float y, const float* b, int form) {
  float dx = fmaxz(fmaxz(fsub(b[0], x), fsub(x, b[1])), 0.0f);
  float dy = fmaxz(fmaxz(fsub(b[2], y), fsub(y, b[3])), 0.0f);
  return sq2(dx, dy, form);
}

/* dbscan_cuda.cu:190-194 */
static inline float box_box_d2(const float* a, const float* b, int form) {
  float dx = fmaxz(fmaxz(fsub(b[0], a[1]), fsub(a[0], b[1])), 0.0f);
  float dy = fmaxz(fmaxz(fsub(b[2], a[3]), fsub(a[2], b[3])), 0.0f);
  return sq2(dx, dy, form);
}

/* static_cast<int32_t>(floorf(v)) on the device: round toward -inf,
 * saturating at the int32 range, NaN -> 0 (cvt.rmi.s32.f32 semantics). */
static inline int32_t floor_to_i32(float v) {
  if (isnan(v)) return 0;
  float f = floorf(v);
  if (f >= 2147483648.0f) return INT32_MAX;
  if (f < -2147483648.0f) return INT32_MIN;
  return (int32_t)f;
}

/* dbscan_cuda.cu:47-50 */
static inline uint64_t pack_key(int32_t kx, int32_t ky) {
  return ((uint64_t)(uint32_t)kx << 32) | (uint64_t)(uint32_t)ky;
}

/* Stable LSD radix sort of u64 keys carrying int32 indices; digits whose
 * value is the same for every key are skipped. Same order as the stable
 * ascending unsigned sort of dbscan_cuda.cu:582-586. */
static int sort_keys(uint64_t* keys, int32_t* idx, int64_t n) {
  uint64_t* k2 = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)n);
  int32_t* i2 = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
  if (!k2 || !i2) { free(k2); free(i2); return -1; }
  uint64_t* ka = keys; int32_t* ia = idx; uint64_t* kb = k2; int32_t* ib = i2;
  for (int shift = 0; shift < 64; shift += 8) {
    int64_t cnt[257];
    memset(cnt, 0, sizeof(cnt));
    for (int64_t i = 0; i < n; ++i) cnt[((ka[i] >> shift) & 0xFF) + 1]++;
    int constant = 0;
    for (int d = 0; d < 256; ++d) if (cnt[d + 1] == n) constant = 1;
    if (constant) continue;
    for (int d = 0; d < 256; ++d) cnt[d + 1] += cnt[d];
    for (int64_t i = 0; i < n; ++i) {
      int d = (int)((ka[i] >> shift) & 0xFF);
      int64_t p = cnt[d]++;
      kb[p] = ka[i]; ib[p] = ia[i];
    }
    uint64_t* tk = ka; ka = kb; kb = tk;
    int32_t* ti = ia; ia = ib; ib = ti;
  }
  if (ka != keys) {
    memcpy(keys, ka, sizeof(uint64_t) * (size_t)n);
    memcpy(idx, ia, sizeof(int32_t) * (size_t)n);
  }
  free(k2); free(i2);
  return 0;
}

/* dbscan_cuda.cu:125-135 */
static int32_t binsearch_cell(const uint64_t* keys, int32_t num_cells, uint64_t target) {
  int32_t lo = 0, hi = num_cells;
  while (lo < hi) {
    int32_t mid = (int32_t)(((int64_t)lo + hi) >> 1);
    if (keys[mid] < target) lo = mid + 1; else hi = mid;
  }
  if (lo < num_cells && keys[lo] == target) return lo;
  return -1;
}

static int32_t uf_find(int32_t* uf, int32_t x) {
  while (uf[x] != x) { uf[x] = uf[uf[x]]; x = uf[x]; }
  return x;
}

/*
 * Runs the whole pipeline. Returns num_cells (>= 0) or -1 on allocation
 * failure. `forms` holds NUM_SITES entries (NULL: all FORM_FMA_X).
 * Optional outputs (NULL to skip) follow the 11-tensor layout of
 * dbscan2d_cuda_debug (dbscan_cuda.cu:777-789): keys_sorted[n], perm[n],
 * xs[n], ys[n], is_core[n], cell_start[n+1], cluster_id[n], uf[n],
 * pre_border[n], final_sorted[n]; cell-sized arrays need capacity n (+1).
 */
int64_t oracle_dbscan2d(const float* X, int64_t n64, double eps, int32_t ms,
                        const int32_t* forms_in, int32_t* labels,
                        uint64_t* o_keys, int32_t* o_perm, float* o_xs, float* o_ys,
                        uint8_t* o_core, int32_t* o_cell_start, int32_t* o_cluster,
                        int32_t* o_uf, int32_t* o_pre, int32_t* o_final) {
  int forms[NUM_SITES];
  for (int s = 0; s < NUM_SITES; ++s) forms[s] = forms_in ? forms_in[s] : FORM_FMA_X;
  if (n64 <= 0) return 0;
  const int32_t n = (int32_t)n64;
  const float fl_eps = (float)eps;
  const float inv_r = sqrtf(2.0f) / fl_eps;
  const float eps_sq = fl_eps * fl_eps;

  int64_t ret = -1;
  uint64_t* keys = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)n);
  int32_t* perm = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
  float* xs = (float*)malloc(sizeof(float) * (size_t)n);
  float* ys = (float*)malloc(sizeof(float) * (size_t)n);
  int32_t* point_cell = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
  int32_t* cell_start = (int32_t*)malloc(sizeof(int32_t) * ((size_t)n + 1));
  uint64_t* cell_keys = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)n);
  uint8_t* is_core = (uint8_t*)calloc((size_t)n, 1);
  int32_t* sl = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
  int32_t* slf = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
  float* bbox = NULL; int32_t* ngh = NULL; uint8_t* status = NULL;
  int32_t* uf = NULL; int32_t* rscan = NULL; int32_t* cid = NULL;
  if (!keys || !perm || !xs || !ys || !point_cell || !cell_start || !cell_keys ||
      !is_core || !sl || !slf) goto done;

  /* stage 1 */
  for (int32_t i = 0; i < n; ++i) {
    int32_t kx = floor_to_i32(fmul(X[2 * (int64_t)i], inv_r));
    int32_t ky = floor_to_i32(fmul(X[2 * (int64_t)i + 1], inv_r));
    keys[i] = pack_key(kx, ky);
    perm[i] = i;
  }
  /* stage 2 */
  if (sort_keys(keys, perm, n) != 0) goto done;
  for (int32_t i = 0; i < n; ++i) {
    xs[i] = X[2 * (int64_t)perm[i]];
    ys[i] = X[2 * (int64_t)perm[i] + 1];
  }
  /* stage 3 */
  int32_t C = 0;
  for (int32_t i = 0; i < n; ++i) {
    if (i == 0 || keys[i] != keys[i - 1]) { cell_start[C] = i; cell_keys[C] = keys[i]; ++C; }
    point_cell[i] = C - 1;
  }
  cell_start[C] = n;
  bbox = (float*)malloc(sizeof(float) * 4 * (size_t)C);
  ngh = (int32_t*)malloc(sizeof(int32_t) * 25 * (size_t)C);
  status = (uint8_t*)malloc((size_t)C);
  uf = (int32_t*)malloc(sizeof(int32_t) * (size_t)C);
  rscan = (int32_t*)malloc(sizeof(int32_t) * (size_t)C);
  cid = (int32_t*)malloc(sizeof(int32_t) * (size_t)C);
  if (!bbox || !ngh || !status || !uf || !rscan || !cid) goto done;
  for (int32_t c = 0; c < C; ++c) {
    int32_t s = cell_start[c], e = cell_start[c + 1];
    float xmin = xs[s], xmax = xs[s], ymin = ys[s], ymax = ys[s];
    for (int32_t i = s + 1; i < e; ++i) {
      xmin = fminz(xmin, xs[i]); xmax = fmaxz(xmax, xs[i]);
      ymin = fminz(ymin, ys[i]); ymax = fmaxz(ymax, ys[i]);
    }
    bbox[4 * (size_t)c + 0] = xmin; bbox[4 * (size_t)c + 1] = xmax;
    bbox[4 * (size_t)c + 2] = ymin; bbox[4 * (size_t)c + 3] = ymax;
  }
  /* stage 4: offsets off = (dx+2)*5 + (dy+2), int32 arithmetic wraps */
  for (int32_t c = 0; c < C; ++c) {
    int32_t kx = (int32_t)(uint32_t)(cell_keys[c] >> 32);
    int32_t ky = (int32_t)(uint32_t)cell_keys[c];
    for (int off = 0; off < 25; ++off) {
      int32_t dx = off / 5 - 2, dy = off % 5 - 2;
      uint64_t t = pack_key((int32_t)((uint32_t)kx + (uint32_t)dx),
                            (int32_t)((uint32_t)ky + (uint32_t)dy));
      ngh[25 * (size_t)c + off] = binsearch_cell(cell_keys, C, t);
    }
  }
  /* stage 5: pass 1 (full cells), pass 2 (per-point count), cell status */
  for (int32_t c = 0; c < C; ++c)
    if (cell_start[c + 1] - cell_start[c] >= ms)
      for (int32_t i = cell_start[c]; i < cell_start[c + 1]; ++i) is_core[i] = 1;
  for (int32_t i = 0; i < n; ++i) {
    if (is_core[i]) continue;
    const int32_t* row = ngh + 25 * (size_t)point_cell[i];
    float xi = xs[i], yi = ys[i];
    int32_t cnt = 0;
    for (int off = 0; off < 25; ++off) {
      int32_t nc = row[off];
      if (nc < 0) continue;
      if (off == 12) {
        cnt += cell_start[nc + 1] - cell_start[nc];
        if (cnt >= ms) break;
      } else {
        if (!fle(point_box_d2(xi, yi, bbox + 4 * (size_t)nc, forms[SITE_CORE_BOX]), eps_sq)) continue;
        for (int32_t j = cell_start[nc]; j < cell_start[nc + 1]; ++j) {
          float ex = fsub(xs[j], xi), ey = fsub(ys[j], yi);
          if (fle(sq2(ex, ey, forms[SITE_CORE_PAIR]), eps_sq)) ++cnt;
        }
        if (cnt >= ms) break;
      }
    }
    if (cnt >= ms) is_core[i] = 1;
  }
  for (int32_t c = 0; c < C; ++c) {
    int any = 0, all = cell_start[c + 1] > cell_start[c];
    for (int32_t j = cell_start[c]; j < cell_start[c + 1]; ++j) {
      if (is_core[j]) any = 1; else all = 0;
    }
    status[c] = (uint8_t)(!any ? 0 : (all ? 2 : 1));
  }
  /* stage 6: components of the cell graph; root = smallest cell index */
  for (int32_t c = 0; c < C; ++c) uf[c] = c;
  for (int32_t c = 0; c < C; ++c) {
    if (status[c] == 0) continue;
    const float* bb_c = bbox + 4 * (size_t)c;
    for (int off = 0; off < 25; ++off) {
      if (off == 12) continue;
      int32_t nc = ngh[25 * (size_t)c + off];
      if (nc <= c || status[nc] == 0) continue;
      if (uf_find(uf, c) == uf_find(uf, nc)) continue;
      const float* bb_n = bbox + 4 * (size_t)nc;
      if (!fle(box_box_d2(bb_c, bb_n, forms[SITE_UNITE_BB]), eps_sq)) continue;
      int found = 0;
      for (int32_t i = cell_start[c]; i < cell_start[c + 1] && !found; ++i) {
        if (!is_core[i]) continue;
        float xi = xs[i], yi = ys[i];
        if (!fle(point_box_d2(xi, yi, bb_n, forms[SITE_UNITE_BOX]), eps_sq)) continue;
        for (int32_t j = cell_start[nc]; j < cell_start[nc + 1]; ++j) {
          if (!is_core[j]) continue;
          float ex = fsub(xs[j], xi), ey = fsub(ys[j], yi);
          if (fle(sq2(ex, ey, forms[SITE_UNITE_PAIR]), eps_sq)) { found = 1; break; }
        }
      }
      if (found) {
        int32_t a = uf_find(uf, c), b = uf_find(uf, nc);
        if (a != b) { if (a < b) uf[b] = a; else uf[a] = b; }
      }
    }
  }
  for (int32_t c = 0; c < C; ++c) uf[c] = uf_find(uf, c);
  /* stage 7 */
  int32_t run = 0;
  for (int32_t c = 0; c < C; ++c) {
    rscan[c] = run;
    run += (uf[c] == c && status[c] != 0) ? 1 : 0;
  }
  for (int32_t c = 0; c < C; ++c) cid[c] = status[c] == 0 ? ORACLE_NOISE : rscan[uf[c]];
  /* stage 8 */
  for (int32_t i = 0; i < n; ++i) sl[i] = is_core[i] ? cid[point_cell[i]] : ORACLE_NOISE;
  /* stage 9 */
  for (int32_t i = 0; i < n; ++i) {
    if (is_core[i]) { slf[i] = sl[i]; continue; }
    const int32_t* row = ngh + 25 * (size_t)point_cell[i];
    float xi = xs[i], yi = ys[i];
    float best_d2 = eps_sq + 1.0f;
    int32_t best_perm = INT32_MAX, best_lab = ORACLE_NOISE;
    for (int off = 0; off < 25; ++off) {
      int32_t nc = row[off];
      if (nc < 0 || status[nc] == 0) continue;
      if (!fle(point_box_d2(xi, yi, bbox + 4 * (size_t)nc, forms[SITE_BORDER_BOX]), eps_sq)) continue;
      for (int32_t j = cell_start[nc]; j < cell_start[nc + 1]; ++j) {
        if (!is_core[j]) continue;
        float ex = fsub(xs[j], xi), ey = fsub(ys[j], yi);
        float d2 = sq2(ex, ey, forms[SITE_BORDER_PAIR]);
        if (!fle(d2, eps_sq)) continue;
        int32_t pj = perm[j];
        if (flt(d2, best_d2) || (feq(d2, best_d2) && pj < best_perm)) {
          best_d2 = d2; best_perm = pj; best_lab = sl[j];
        }
      }
    }
    slf[i] = best_lab;
  }
  /* stage 10 */
  for (int32_t i = 0; i < n; ++i) labels[i] = ORACLE_NOISE;
  for (int32_t i = 0; i < n; ++i) labels[perm[i]] = slf[i];

  if (o_keys) memcpy(o_keys, keys, sizeof(uint64_t) * (size_t)n);
  if (o_perm) memcpy(o_perm, perm, sizeof(int32_t) * (size_t)n);
  if (o_xs) memcpy(o_xs, xs, sizeof(float) * (size_t)n);
  if (o_ys) memcpy(o_ys, ys, sizeof(float) * (size_t)n);
  if (o_core) memcpy(o_core, is_core, (size_t)n);
  if (o_cell_start) memcpy(o_cell_start, cell_start, sizeof(int32_t) * ((size_t)C + 1));
  if (o_cluster) memcpy(o_cluster, cid, sizeof(int32_t) * (size_t)C);
  if (o_uf) memcpy(o_uf, uf, sizeof(int32_t) * (size_t)C);
  if (o_pre) memcpy(o_pre, sl, sizeof(int32_t) * (size_t)n);
  if (o_final) memcpy(o_final, slf, sizeof(int32_t) * (size_t)n);
  ret = C;

done:
  free(keys); free(perm); free(xs); free(ys); free(point_cell); free(cell_start);
  free(cell_keys); free(is_core); free(sl); free(slf); free(bbox); free(ngh);
  free(status); free(uf); free(rscan); free(cid);
  return ret;
}

/* Squared distance of one pair in a given form, with the device's flush and
 * subtraction order (ex = xj - xi). Exposed so tests can build inputs on
 * which the forms disagree. */
float oracle_pair_d2(float xi, float yi, float xj, float yj, int32_t form) {
  return sq2(fsub(xj, xi), fsub(yj, yi), form);
}

/* Vectorised pair_d2 for probe construction: out[k] = d2 of pair k. */
void oracle_pair_d2_batch(const float* a, const float* b, int64_t count, int32_t form, float* out) {
  for (int64_t k = 0; k < count; ++k)
    out[k] = oracle_pair_d2(a[2 * k], a[2 * k + 1], b[2 * k], b[2 * k + 1], form);
}
