/*
 * TEST INFRASTRUCTURE ONLY (the oracle's graph generators, multi-threaded).
 *
 * The same seeded RMAT / uniform / grid graphs as oracle/graphgen.py (the
 * numpy restatement, which states the definitions) and as the CUDA
 * library's device generator, built on the host cores with OpenMP.  It lets
 * the CPU legs of the benchmark build a scale-24 graph in seconds without
 * loading the product library: the reference's bfs then runs on a graph that
 * no product code touched.  Tests check it bit for bit against the numpy
 * restatement.
 *
 * CSR clean-up as in NWGraph's edge-list pipeline: both directions of every
 * undirected pair (io/mmio.hpp:96-100 for symmetric files), self-loops
 * dropped (build.hpp:427-444), rows sorted and deduplicated (build.hpp:58-70,
 * 344-355), rows filled in neighbour order (build.hpp:210-266).
 *
 * Pipeline: pass 1 generates every pair and counts both endpoints' rows;
 * pass 2 generates the pairs again and scatters the neighbours; then each
 * row is sorted and deduplicated in place and the rows are compacted into
 * the output.  Generating twice keeps the host memory at 8 bytes per
 * directed entry.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include <omp.h>

#define GOLDEN 0x9E3779B97F4A7C15ull
#define MIX1 0xBF58476D1CE4E5B9ull
#define MIX2 0x94D049BB133111EBull

enum { STREAM_RMAT = 1, STREAM_PERM = 2, STREAM_UNIFORM = 3, STREAM_GRID = 4 };
enum { KIND_RMAT = 0, KIND_UNIFORM = 1, KIND_GRID = 2 };

static inline uint64_t splitmix64(uint64_t x) {
  uint64_t z = x + GOLDEN;
  z = (z ^ (z >> 30)) * MIX1;
  z = (z ^ (z >> 27)) * MIX2;
  return z ^ (z >> 31);
}

static inline uint64_t lemire(uint64_t h, uint64_t n) { return ((h >> 32) * n) >> 32; }

typedef struct {
  int kind;
  uint64_t n;
  uint64_t pairs;
  uint64_t key_rmat, key_uniform, key_grid; /* splitmix64(seed) ^ (stream << 56) */
  /* RMAT */
  int scale;
  uint64_t ta, tab, tabc;
  uint64_t perm_k[3], perm_c[3];
  /* grid */
  uint64_t width, height, grid_right, grid_edges;
} spec_t;

static inline uint64_t permute(const spec_t* s, uint64_t x) {
  const uint64_t mask = (s->scale >= 64) ? ~0ull : ((1ull << s->scale) - 1);
  const int sh = (s->scale + 1) >> 1;
  for (int r = 0; r < 3; r++) {
    x = (x * s->perm_k[r] + s->perm_c[r]) & mask;
    x ^= x >> sh;
  }
  return x;
}

/* The i-th undirected pair of the graph (before symmetrization). */
static inline void pair_at(const spec_t* s, uint64_t i, uint64_t* pu, uint64_t* pv) {
  if (s->kind == KIND_RMAT) {
    const uint64_t words = (uint64_t)((s->scale + 1) >> 1);
    uint64_t u = 0, v = 0, w = 0;
    for (int lvl = 0; lvl < s->scale; lvl++) {
      if (!(lvl & 1)) w = splitmix64((i * words + (uint64_t)(lvl >> 1)) ^ s->key_rmat);
      const uint64_t t = (lvl & 1) ? (w >> 32) : (w & 0xFFFFFFFFull);
      const uint64_t ub = t >= s->tab;
      const uint64_t vb = ((t >= s->ta) && (t < s->tab)) || (t >= s->tabc);
      u = (u << 1) | ub;
      v = (v << 1) | vb;
    }
    *pu = permute(s, u);
    *pv = permute(s, v);
  } else if (s->kind == KIND_UNIFORM) {
    *pu = lemire(splitmix64((2 * i) ^ s->key_uniform), s->n);
    *pv = lemire(splitmix64((2 * i + 1) ^ s->key_uniform), s->n);
  } else {
    if (i < s->grid_right) { /* right neighbours: row y, columns 0..w-2 */
      const uint64_t y = i / (s->width - 1), x = i % (s->width - 1);
      *pu = y * s->width + x;
      *pv = *pu + 1;
    } else if (i < s->grid_edges) { /* down neighbours: rows 0..h-2 */
      const uint64_t j = i - s->grid_right;
      *pu = j;
      *pv = j + s->width;
    } else { /* shortcuts */
      const uint64_t j = i - s->grid_edges;
      *pu = lemire(splitmix64((2 * j) ^ s->key_grid), s->n);
      *pv = lemire(splitmix64((2 * j + 1) ^ s->key_grid), s->n);
    }
  }
}

static int cmp_u32(const void* a, const void* b) {
  const uint32_t x = *(const uint32_t*)a, y = *(const uint32_t*)b;
  return (x > y) - (x < y);
}

static uint64_t sort_dedup(uint32_t* r, uint64_t len) {
  if (len < 2) return len;
  if (len <= 32) {
    for (uint64_t i = 1; i < len; i++) {
      uint32_t x = r[i];
      uint64_t j = i;
      while (j > 0 && r[j - 1] > x) {
        r[j] = r[j - 1];
        j--;
      }
      r[j] = x;
    }
  } else {
    qsort(r, len, sizeof(uint32_t), cmp_u32);
  }
  uint64_t k = 1;
  for (uint64_t i = 1; i < len; i++)
    if (r[i] != r[k - 1]) r[k++] = r[i];
  return k;
}

/* Number of undirected pairs the spec generates (2x is the capacity that
 * tmp and cols need). */
static int make_spec(spec_t* s, int kind, uint64_t a0, uint64_t a1, uint64_t a2, uint64_t seed, uint32_t ta,
                     uint32_t tab, uint32_t tabc) {
  memset(s, 0, sizeof(*s));
  s->kind = kind;
  const uint64_t key = splitmix64(seed);
  s->key_rmat = key ^ ((uint64_t)STREAM_RMAT << 56);
  s->key_uniform = key ^ ((uint64_t)STREAM_UNIFORM << 56);
  s->key_grid = key ^ ((uint64_t)STREAM_GRID << 56);
  if (kind == KIND_RMAT) { /* a0 = scale, a1 = edge factor */
    if (a0 < 1 || a0 > 32) return -1;
    s->scale = (int)a0;
    s->n = 1ull << a0;
    s->pairs = a1 << a0;
    s->ta = ta;
    s->tab = tab;
    s->tabc = tabc;
    const uint64_t pk = key ^ ((uint64_t)STREAM_PERM << 56);
    for (int r = 0; r < 3; r++) {
      s->perm_k[r] = splitmix64((uint64_t)(2 * r) ^ pk) | 1;
      s->perm_c[r] = splitmix64((uint64_t)(2 * r + 1) ^ pk);
    }
  } else if (kind == KIND_UNIFORM) { /* a0 = n, a1 = average degree */
    if (a0 < 1 || a0 > 0xFFFFFFFFull) return -1;
    s->n = a0;
    s->pairs = (a0 * a1) / 2;
  } else if (kind == KIND_GRID) { /* a0 = width, a1 = height, a2 = shortcut percent */
    if (a0 < 2 || a1 < 2 || a0 * a1 > 0xFFFFFFFFull) return -1;
    s->width = a0;
    s->height = a1;
    s->n = a0 * a1;
    s->grid_right = a1 * (a0 - 1);
    s->grid_edges = s->grid_right + (a1 - 1) * a0;
    s->pairs = s->grid_edges + (s->grid_edges * a2) / 100;
  } else {
    return -1;
  }
  return 0;
}

/* Capacity (directed entries before dedup) that nwggen_csr needs in tmp and
 * cols, or 0 for a bad spec. */
uint64_t nwggen_capacity(int kind, uint64_t a0, uint64_t a1, uint64_t a2) {
  spec_t s;
  if (make_spec(&s, kind, a0, a1, a2, 0, 0, 0, 0) != 0) return 0;
  return 2 * s.pairs;
}

uint64_t nwggen_vertices(int kind, uint64_t a0, uint64_t a1, uint64_t a2) {
  spec_t s;
  if (make_spec(&s, kind, a0, a1, a2, 0, 0, 0, 0) != 0) return 0;
  return s.n;
}

/* Builds the CSR: off[n+1] (uint64), cols[0..m) (uint32, rows sorted and
 * deduplicated); tmp and cols hold `cap` entries each (nwggen_capacity).
 * Returns m, or a negative error.  threads <= 0 uses OpenMP's default. */
int64_t nwggen_csr(int kind, uint64_t a0, uint64_t a1, uint64_t a2, uint64_t seed, uint32_t ta, uint32_t tab,
                   uint32_t tabc, int threads, uint64_t* off, uint32_t* tmp, uint32_t* cols, uint64_t cap) {
  spec_t s;
  if (make_spec(&s, kind, a0, a1, a2, seed, ta, tab, tabc) != 0) return -1;
  if (cap < 2 * s.pairs) return -2;
  const uint64_t n = s.n;
  const uint64_t P = s.pairs;
  if (threads > 0) omp_set_num_threads(threads);
  const int T = omp_get_max_threads();
  /* hist[t * n + u]: entries thread t adds to row u, then its first slot in
   * that row.  Each thread owns a fixed slice of the pairs in both passes,
   * so the two passes agree and no thread writes another's slots. */
  uint32_t* hist = (uint32_t*)calloc((size_t)T * n, sizeof(uint32_t));
  uint64_t* cnt = (uint64_t*)malloc((n + 1) * sizeof(uint64_t));
  if (!hist || !cnt) {
    free(hist);
    free(cnt);
    return -3;
  }

  /* pass 1: row lengths per thread (both directions, self-loops dropped) */
#pragma omp parallel num_threads(T)
  {
    const int t = omp_get_thread_num();
    uint32_t* h = hist + (size_t)t * n;
    const uint64_t lo = P * (uint64_t)t / (uint64_t)T, hi = P * (uint64_t)(t + 1) / (uint64_t)T;
    for (uint64_t i = lo; i < hi; i++) {
      uint64_t u, v;
      pair_at(&s, i, &u, &v);
      if (u == v) continue;
      h[u]++;
      h[v]++;
    }
  }
  /* each thread's first slot within each row; cnt[u] = row length */
#pragma omp parallel for schedule(static, 1 << 14) num_threads(T)
  for (int64_t u = 0; u < (int64_t)n; u++) {
    uint32_t acc = 0;
    for (int t = 0; t < T; t++) {
      const uint32_t c = hist[(size_t)t * n + u];
      hist[(size_t)t * n + u] = acc;
      acc += c;
    }
    cnt[u] = acc;
  }
  uint64_t acc = 0;
  for (uint64_t u = 0; u < n; u++) {
    off[u] = acc;
    acc += cnt[u];
  }
  off[n] = acc;
  /* pass 2: scatter */
#pragma omp parallel num_threads(T)
  {
    const int t = omp_get_thread_num();
    uint32_t* h = hist + (size_t)t * n;
    const uint64_t lo = P * (uint64_t)t / (uint64_t)T, hi = P * (uint64_t)(t + 1) / (uint64_t)T;
    for (uint64_t i = lo; i < hi; i++) {
      uint64_t u, v;
      pair_at(&s, i, &u, &v);
      if (u == v) continue;
      tmp[off[u] + h[u]++] = (uint32_t)v;
      tmp[off[v] + h[v]++] = (uint32_t)u;
    }
  }
  free(hist);
  /* sort and deduplicate each row in place; cnt[u] = its new length */
#pragma omp parallel for schedule(dynamic, 4096)
  for (int64_t u = 0; u < (int64_t)n; u++) cnt[u] = sort_dedup(tmp + off[u], off[u + 1] - off[u]);
  /* compact into cols and rewrite off */
  acc = 0;
  for (uint64_t u = 0; u < n; u++) {
    const uint64_t c = cnt[u];
    cnt[u] = acc; /* new start */
    acc += c;
  }
  cnt[n] = acc;
#pragma omp parallel for schedule(dynamic, 4096)
  for (int64_t u = 0; u < (int64_t)n; u++) memcpy(cols + cnt[u], tmp + off[u], (cnt[u + 1] - cnt[u]) * 4);
  memcpy(off, cnt, (n + 1) * sizeof(uint64_t));
  free(cnt);
  return (int64_t)acc;
}
