/*
 * tc_oracle.c -- CPU restatement of bbTC's counting path.  TEST
 * INFRASTRUCTURE ONLY: the parity checker for tests/, the smoke check and the
 * CPU baseline of bench.py.  The library never links or calls it.
 *
 * It follows the reference step by step (paths inside the bbTC project):
 *   block CSR   src/data_structures/block_csr.cpp:288-376 (CSRtoBCSR):
 *               sparse_tiles_[t] = first row slot of tile t (tiles row-major,
 *               each P x (height of its row part) slots); rows_ = per-row
 *               counts by tile, one running scan, global offsets into cols_;
 *               cols_ = tile-local column ids.
 *   tile degree block_csr.cpp:258-284 (tile_deg = nnz / height),
 *               IsDense: tile_deg > 10000 (block_csr.h:35, block_csr.cpp:209-212)
 *   task list   include/utils/tasks.hpp:7-17, (i <= j <= k) -> {ij, jk, ik}
 *   task skip   src/triangle_counting/bb_tc.cpp:124-129 (any tile_deg == 0)
 *   sparse task src/triangle_counting/cpu_sparse_kernel.cpp:41-59, merge
 *               ListIntersect with the early exits of :3-39
 *   dense task  src/triangle_counting/cpu_dense_kernel.cpp:24-51, stamped
 *               hashmap for rows of >= 4 entries, merge below (:43-47)
 * Tasks are independent; the total is their sum, so the OpenMP loop over
 * tasks returns the same count as the reference's work queue.
 *
 * Pinned against the reference itself: tests compare it with oracle/_ref
 * (the reference's own headers, compiled by oracle/Makefile) on seeded graphs,
 * and with known answers (complete graphs, wheels, bipartite graphs).
 */
#include <omp.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
  uint32_t P, n;
  uint32_t* cuts;          /* P+1 */
  uint64_t* sparse_tiles;  /* P*P+1 row-slot offsets */
  uint32_t* rows;          /* row slots: global offsets into cols */
  uint32_t* cols;          /* tile-local column ids */
  float* tile_deg;         /* P*P */
  uint64_t nslots;
} oracle_bcsr;

static void bcsr_free(oracle_bcsr* b) {
  free(b->cuts);
  free(b->sparse_tiles);
  free(b->rows);
  free(b->cols);
  free(b->tile_deg);
}

/* CSRtoBCSR (block_csr.cpp:288-376) and ComputeTileProps (:258-284). */
static int bcsr_build(oracle_bcsr* b, uint32_t n, const uint32_t* indptr, const uint32_t* indices,
                      const uint32_t* cuts, uint32_t P) {
  memset(b, 0, sizeof(*b));
  b->P = P;
  b->n = n;
  const uint64_t T = (uint64_t)P * P;
  b->cuts = (uint32_t*)malloc((P + 1) * sizeof(uint32_t));
  b->sparse_tiles = (uint64_t*)malloc((T + 1) * sizeof(uint64_t));
  b->tile_deg = (float*)malloc(T * sizeof(float));
  if (!b->cuts || !b->sparse_tiles || !b->tile_deg) return -2;
  memcpy(b->cuts, cuts, (P + 1) * sizeof(uint32_t));
  b->sparse_tiles[0] = 0;
  for (uint32_t i = 0; i < P; i++)
    for (uint32_t j = 0; j < P; j++)
      b->sparse_tiles[i * P + j + 1] = b->sparse_tiles[i * P + j] + (cuts[i + 1] - cuts[i]);
  b->nslots = b->sparse_tiles[T] + 1;
  b->rows = (uint32_t*)calloc(b->nslots, sizeof(uint32_t));
  b->cols = (uint32_t*)malloc((indptr[n] ? indptr[n] : 1) * sizeof(uint32_t));
  if (!b->rows || !b->cols) return -2;
  /* per-row count by tile column: slot (tile start + local row + 1) */
#pragma omp parallel for schedule(dynamic, 2048)
  for (int64_t u = 0; u < (int64_t)n; u++) {
    uint32_t x = 0, y = 0;
    while ((uint32_t)u >= cuts[y + 1]) y++;
    for (uint32_t v = indptr[u]; v < indptr[u + 1]; v++) {
      while (indices[v] >= cuts[x + 1]) x++;
      b->rows[b->sparse_tiles[(uint64_t)y * P + x] + (u - cuts[y]) + 1] += 1;
    }
  }
  for (uint64_t i = 1; i < b->nslots; i++) b->rows[i] += b->rows[i - 1];
  /* scatter tile-local columns */
#pragma omp parallel for schedule(dynamic, 2048)
  for (int64_t u = 0; u < (int64_t)n; u++) {
    uint32_t x = 0, y = 0;
    while ((uint32_t)u >= cuts[y + 1]) y++;
    uint64_t pos = b->rows[b->sparse_tiles[(uint64_t)y * P] + (u - cuts[y])];
    for (uint32_t v = indptr[u]; v < indptr[u + 1]; v++) {
      while (indices[v] >= cuts[x + 1]) {
        x++;
        pos = b->rows[b->sparse_tiles[(uint64_t)y * P + x] + (u - cuts[y])];
      }
      b->cols[pos++] = indices[v] - cuts[x];
    }
  }
  for (uint64_t t = 0; t < T; t++) {
    const uint64_t s0 = b->sparse_tiles[t], s1 = b->sparse_tiles[t + 1];
    const uint64_t nnz = b->rows[s1] - b->rows[s0];
    b->tile_deg[t] = (float)nnz / (float)(s1 - s0);
  }
  return 0;
}

static uint64_t tile_nnz(const oracle_bcsr* b, uint64_t t) {
  return b->rows[b->sparse_tiles[t + 1]] - b->rows[b->sparse_tiles[t]];
}

/* ListIntersect (cpu_sparse_kernel.cpp:3-39). */
static uint64_t list_intersect(const oracle_bcsr* b, uint64_t ab_src, uint64_t bc_src, uint64_t ac_src,
                               uint32_t f_i) {
  const uint32_t* rows = b->rows;
  const uint32_t* cols = b->cols;
  uint64_t n = 0;
  const uint32_t r_i = rows[ac_src + f_i + 1];
  for (uint32_t i = rows[ab_src + f_i]; i < rows[ab_src + f_i + 1]; i++) {
    const uint32_t bb = cols[i];
    uint32_t l_j = rows[bc_src + bb];
    const uint32_t r_j = rows[bc_src + bb + 1];
    uint32_t l_i = rows[ac_src + f_i];
    while (l_i < r_i && l_j < r_j) {
      if (cols[l_i] == cols[l_j]) {
        ++l_i;
        ++l_j;
        ++n;
      } else if (cols[l_i] < cols[l_j]) {
        if (cols[l_j] > cols[r_i - 1]) break;
        ++l_i;
      } else {
        if (cols[l_i] > cols[r_j - 1]) break;
        ++l_j;
      }
    }
  }
  return n;
}

/* TrianglesInASparseTask (cpu_sparse_kernel.cpp:41-59). */
static uint64_t sparse_task(const oracle_bcsr* b, uint64_t ab, uint64_t bc, uint64_t ac) {
  const uint64_t height = b->sparse_tiles[ab + 1] - b->sparse_tiles[ab];
  const uint64_t ab_src = b->sparse_tiles[ab], bc_src = b->sparse_tiles[bc], ac_src = b->sparse_tiles[ac];
  uint64_t n = 0;
  for (uint32_t f_i = 0; f_i < height; f_i++) {
    if (b->rows[ac_src + f_i + 1] == b->rows[ac_src + f_i]) continue;
    n += list_intersect(b, ab_src, bc_src, ac_src, f_i);
  }
  return n;
}

/* TrianglesInADenseTask + ListIntersectUsingHMap (cpu_dense_kernel.cpp:3-51). */
static uint64_t dense_task(const oracle_bcsr* b, uint64_t ab, uint64_t bc, uint64_t ac, uint32_t* hmap) {
  const uint32_t* rows = b->rows;
  const uint32_t* cols = b->cols;
  const uint64_t height = b->sparse_tiles[ab + 1] - b->sparse_tiles[ab];
  const uint64_t ab_src = b->sparse_tiles[ab], bc_src = b->sparse_tiles[bc], ac_src = b->sparse_tiles[ac];
  const uint32_t width = b->cuts[ac % b->P + 1] - b->cuts[ac % b->P];
  for (uint32_t i = 0; i < width; i++) hmap[i] = 0x7fffffffu;
  uint64_t n = 0;
  for (uint32_t f_i = 0; f_i < height; f_i++) {
    if (rows[ac_src + f_i + 1] == rows[ac_src + f_i]) continue;
    if (rows[ab_src + f_i + 1] - rows[ab_src + f_i] < 4) {
      n += list_intersect(b, ab_src, bc_src, ac_src, f_i);
      continue;
    }
    for (uint32_t i = rows[ac_src + f_i]; i < rows[ac_src + f_i + 1]; i++) hmap[cols[i]] = f_i;
    for (uint32_t i = rows[ab_src + f_i]; i < rows[ab_src + f_i + 1]; i++) {
      const uint32_t bb = cols[i];
      for (uint32_t j = rows[bc_src + bb]; j < rows[bc_src + bb + 1]; j++) n += (hmap[cols[j]] == f_i);
    }
  }
  return n;
}

/* Count triangles: the reference's CPU path over the whole TaskList(P).
 * Returns 0 on success; *out receives the count.  nthreads <= 0 uses the
 * OpenMP default. */
int oracle_count(uint32_t n, const uint32_t* indptr, const uint32_t* indices, const uint32_t* cuts, uint32_t P,
                 int nthreads, uint64_t* out) {
  if (!out || !indptr || !cuts || P < 1) return -1;
  if (nthreads > 0) omp_set_num_threads(nthreads);
  oracle_bcsr b;
  int rc = bcsr_build(&b, n, indptr, indices, cuts, P);
  if (rc) {
    bcsr_free(&b);
    return rc;
  }
  /* HASH_LIMIT = largest width among dense tiles (block_csr.cpp:189-206) */
  uint32_t hash_limit = 1;
  for (uint64_t t = 0; t < (uint64_t)P * P; t++)
    if (b.tile_deg[t] > 10000.0f) {
      const uint32_t w = cuts[t % P + 1] - cuts[t % P];
      if (w > hash_limit) hash_limit = w;
    }
  const uint64_t ntasks = (uint64_t)P * (P + 1) * (P + 2) / 6;
  uint64_t* tl = (uint64_t*)malloc(ntasks * 3 * sizeof(uint64_t));
  uint64_t q = 0;
  for (uint64_t i = 0; i < P; i++)
    for (uint64_t j = i; j < P; j++)
      for (uint64_t k = j; k < P; k++) {
        tl[3 * q] = i * P + j;
        tl[3 * q + 1] = j * P + k;
        tl[3 * q + 2] = i * P + k;
        q++;
      }
  uint64_t total = 0;
  int failed = 0;
#pragma omp parallel reduction(+ : total)
  {
    uint32_t* hmap = (uint32_t*)malloc((size_t)hash_limit * sizeof(uint32_t));
    if (!hmap) {
#pragma omp atomic write
      failed = 1;
    }
#pragma omp for schedule(dynamic, 1)
    for (int64_t t = 0; t < (int64_t)ntasks; t++) {
      if (!hmap) continue;
      const uint64_t ab = tl[3 * t], bc = tl[3 * t + 1], ac = tl[3 * t + 2];
      if (b.tile_deg[bc] == 0.0f || b.tile_deg[ac] == 0.0f || b.tile_deg[ab] == 0.0f) continue;
      if (b.tile_deg[ac] > 10000.0f || b.tile_deg[bc] > 10000.0f || b.tile_deg[ab] > 10000.0f)
        total += dense_task(&b, ab, bc, ac, hmap);
      else
        total += sparse_task(&b, ab, bc, ac);
    }
    free(hmap);
  }
  free(tl);
  bcsr_free(&b);
  if (failed) return -2;
  *out = total;
  return 0;
}

/* Per-tile nnz of the reference layout (GetNNZ, block_csr.cpp:88-92), P*P entries. */
int oracle_tile_nnz(uint32_t n, const uint32_t* indptr, const uint32_t* indices, const uint32_t* cuts, uint32_t P,
                    uint64_t* nnz) {
  oracle_bcsr b;
  int rc = bcsr_build(&b, n, indptr, indices, cuts, P);
  if (!rc)
    for (uint64_t t = 0; t < (uint64_t)P * P; t++) nnz[t] = tile_nnz(&b, t);
  bcsr_free(&b);
  return rc;
}

/* Task sum of one task (ab, bc, ac tile ids), for per-task parity checks. */
int oracle_task_count(uint32_t n, const uint32_t* indptr, const uint32_t* indices, const uint32_t* cuts, uint32_t P,
                      uint32_t ab, uint32_t bc, uint32_t ac, uint64_t* out) {
  oracle_bcsr b;
  int rc = bcsr_build(&b, n, indptr, indices, cuts, P);
  if (!rc) {
    if (b.tile_deg[bc] == 0.0f || b.tile_deg[ac] == 0.0f || b.tile_deg[ab] == 0.0f)
      *out = 0;
    else
      *out = sparse_task(&b, ab, bc, ac);
  }
  bcsr_free(&b);
  return rc;
}
