/*
 * TEST INFRASTRUCTURE ONLY (the oracle).  A plain-C, single-threaded
 * restatement of NWGraph's breadth-first searches, used by tests/ and by
 * bench.py's CPU-baseline leg as the checker.  The product never links it.
 *
 * Functions and the reference lines they restate (paths are relative to the
 * NWGraph source tree):
 *   nwgport_dobfs       nw::graph::bfs(out, in, root, num_bins, alpha, beta),
 *                       include/nwgraph/algorithms/bfs.hpp:160-311.  Records a
 *                       per-step trace of the direction decisions so the GPU's
 *                       device-side decisions can be compared step by step.
 *   nwgport_bfs_depths  level-synchronous BFS depths, the same traversal as the
 *                       serial bfs(graph, root) at bfs.hpp:110-140 and the
 *                       depth pass of BFSVerifier at bfs.hpp:48-65.
 *   nwgport_verify      the checks of BFSVerifier, bfs.hpp:66-97.
 *   nwgport_depths_from_parents
 *                       depth[root] = 0, depth[v] = depth[parent[v]] + 1.
 *   nwgport_msbfs_depths  uint8 depths for a list of sources, each an
 *                       independent single-source BFS (255 = unreached).
 *   nwgport_bc          approximate betweenness centrality over a list of
 *                       sources, the computation of BCVerifier<float, double>
 *                       (include/nwgraph/algorithms/betweenness_centrality.hpp:
 *                       59-115): per source a serial BFS with double path
 *                       counts, then float deltas accumulated from the deepest
 *                       level up; every reached vertex, the source included,
 *                       adds its delta; optional division by the largest score.
 *
 * The pow2(ceil_log2(num_bins)) bin count and the `u % n` binning of
 * bfs.hpp:166,181,287 only order the serial work here; they cannot change
 * depths or the direction decisions.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define NULLV 0xFFFFFFFFu

typedef struct {
  /* one record per outer-loop step of bfs.hpp:184-308 and per inner
   * bottom-up pull of bfs.hpp:205-229 */
  uint32_t cap;       /* capacity of the arrays below (in records) */
  uint32_t steps;     /* records written */
  uint8_t* dir;       /* 0 = top-down step, 1 = bottom-up pull */
  uint64_t* frontier; /* frontier size entering the step */
  uint64_t* found;    /* vertices discovered by the step */
  uint64_t* scout;    /* scout_count after the step (top-down) / awake (bottom-up) */
} nwgport_trace;

static void trace_add(nwgport_trace* t, uint8_t dir, uint64_t frontier, uint64_t found, uint64_t scout) {
  if (!t || t->steps >= t->cap) {
    if (t) t->steps++;
    return;
  }
  t->dir[t->steps]      = dir;
  t->frontier[t->steps] = frontier;
  t->found[t->steps]    = found;
  t->scout[t->steps]    = scout;
  t->steps++;
}

static int ceil_log2_u32(uint32_t v) {
  int l = 31 - __builtin_clz(v);
  return l + ((v & (v - 1)) != 0);
}

/* Returns the number of steps (trace records) or a negative error. */
int64_t nwgport_dobfs(const uint64_t* out_off, const uint32_t* out_col, const uint64_t* in_off, const uint32_t* in_col,
                      uint64_t N, uint32_t root, int num_bins, int alpha, int beta, uint32_t* parents,
                      nwgport_trace* trace) {
  if (root >= N || num_bins <= 0 || alpha <= 0 || beta <= 0) return -1;
  if (!in_off) {
    in_off = out_off;
    in_col = out_col;
  }
  const uint64_t nb = (uint64_t)1 << ceil_log2_u32((uint32_t)num_bins); /* bfs.hpp:166 */
  const uint64_t M  = out_off[N];                                      /* bfs.hpp:168 */
  const uint64_t W  = (N + 63) / 64;

  /* q1/q2: nb bins, each bin a contiguous segment; a vertex enters at most
   * one bin per level, so N slots per bin-set are enough when bins share one
   * array through per-bin counters over a stable split. */
  uint32_t* q1     = (uint32_t*)malloc(sizeof(uint32_t) * (N ? N : 1));
  uint32_t* q2     = (uint32_t*)malloc(sizeof(uint32_t) * (N ? N : 1));
  uint64_t* front  = (uint64_t*)calloc(W ? W : 1, sizeof(uint64_t));
  uint64_t* curr   = (uint64_t*)calloc(W ? W : 1, sizeof(uint64_t));
  uint32_t* tmp    = (uint32_t*)malloc(sizeof(uint32_t) * (N ? N : 1));
  uint64_t* bcount = (uint64_t*)calloc(nb, sizeof(uint64_t));
  if (!q1 || !q2 || !front || !curr || !tmp || !bcount) return -2;
  uint64_t q1n = 0, q2n = 0;

  for (uint64_t i = 0; i < N; ++i) parents[i] = NULLV; /* bfs.hpp:175 */

  uint64_t edges_to_check = M;                                  /* bfs.hpp:177 */
  uint64_t scout_count    = out_off[root + 1] - out_off[root];  /* bfs.hpp:178 */
  parents[root]           = root;                               /* bfs.hpp:180 */
  q1[q1n++]               = root;                               /* bfs.hpp:181 */

  int done = 0;
  while (!done) {
    q2n = 0;
    if (scout_count > edges_to_check / (uint64_t)alpha) { /* bfs.hpp:186 */
      /* queue -> bitmap, awake_count = |q1| (bfs.hpp:199-202) */
      uint64_t awake_count = q1n;
      for (uint64_t i = 0; i < q1n; ++i) curr[q1[i] >> 6] |= 1ull << (q1[i] & 63);
      uint64_t old_awake_count;
      do { /* bfs.hpp:205-229 */
        old_awake_count = awake_count;
        uint64_t* s     = front;
        front           = curr;
        curr            = s;
        memset(curr, 0, W * sizeof(uint64_t));
        awake_count = 0;
        for (uint64_t u = 0; u < N; ++u) {
          if (parents[u] != NULLV) continue;
          for (uint64_t e = in_off[u]; e < in_off[u + 1]; ++e) {
            uint32_t v = in_col[e];
            if (front[v >> 6] & (1ull << (v & 63))) {
              curr[u >> 6] |= 1ull << (u & 63);
              parents[u] = v;
              ++awake_count;
              break;
            }
          }
        }
        trace_add(trace, 1, old_awake_count, awake_count, awake_count);
      } while ((awake_count >= old_awake_count) || (awake_count > N / (uint64_t)beta));

      if (awake_count == 0) { /* bfs.hpp:231-233 */
        done = 1;
        break;
      }
      /* bitmap -> queue in word order (bfs.hpp:235-239); scout = 1 (:241) */
      for (uint64_t w = 0; w < W; ++w) {
        uint64_t x = curr[w];
        while (x) {
          int b      = __builtin_ctzll(x);
          q2[q2n++]  = (uint32_t)(w * 64 + b);
          x &= x - 1;
        }
      }
      scout_count = 1;
    } else {
      /* top-down step, bfs.hpp:242-295 */
      edges_to_check -= scout_count;
      uint64_t frontier = q1n;
      scout_count       = 0;
      /* visit bins in order, entries of a bin in arrival order */
      memset(bcount, 0, nb * sizeof(uint64_t));
      for (uint64_t i = 0; i < q1n; ++i) {
        uint32_t u = q1[i];
        for (uint64_t e = out_off[u]; e < out_off[u + 1]; ++e) {
          uint32_t v = out_col[e];
          if (parents[v] == NULLV) {
            parents[v] = u;
            tmp[q2n++] = v;
            scout_count += out_off[v + 1] - out_off[v];
          }
        }
      }
      /* regroup the next queue by bin u % nb of the discovering vertex is an
       * ordering detail only; keep arrival order */
      memcpy(q2, tmp, q2n * sizeof(uint32_t));
      trace_add(trace, 0, frontier, q2n, scout_count);
    }
    /* termination and swap, bfs.hpp:297-307 */
    done = (q2n == 0);
    uint32_t* s = q1;
    q1          = q2;
    q2          = s;
    q1n         = q2n;
  }

  free(q1);
  free(q2);
  free(front);
  free(curr);
  free(tmp);
  free(bcount);
  return trace ? (int64_t)trace->steps : 0;
}

/* Level-synchronous BFS depths (bfs.hpp:110-140, :48-65).  depth = NULLV for
 * unreached vertices.  Returns the number of levels. */
int64_t nwgport_bfs_depths(const uint64_t* off, const uint32_t* col, uint64_t N, uint32_t root, uint32_t* depth) {
  if (root >= N) return -1;
  uint32_t* q = (uint32_t*)malloc(sizeof(uint32_t) * N);
  if (!q) return -2;
  for (uint64_t i = 0; i < N; ++i) depth[i] = NULLV;
  uint64_t head = 0, tail = 0;
  depth[root] = 0;
  q[tail++]   = root;
  uint32_t maxd = 0;
  while (head < tail) {
    uint32_t u = q[head++];
    for (uint64_t e = off[u]; e < off[u + 1]; ++e) {
      uint32_t v = col[e];
      if (depth[v] == NULLV) {
        depth[v] = depth[u] + 1;
        if (depth[v] > maxd) maxd = depth[v];
        q[tail++] = v;
      }
    }
  }
  free(q);
  return (int64_t)maxd + 1;
}

/* Depths implied by a parent array; NULLV where unreached.  Returns -1 if
 * the parents do not form a tree rooted at root (cycle or dangling parent). */
int64_t nwgport_depths_from_parents(const uint32_t* parents, uint64_t N, uint32_t root, uint32_t* depth) {
  if (root >= N || parents[root] != root) return -1;
  for (uint64_t i = 0; i < N; ++i) depth[i] = NULLV;
  depth[root] = 0;
  uint32_t* stack = (uint32_t*)malloc(sizeof(uint32_t) * N);
  if (!stack) return -2;
  for (uint64_t s = 0; s < N; ++s) {
    if (parents[s] == NULLV || depth[s] != NULLV) continue;
    uint64_t sp = 0;
    uint32_t v  = (uint32_t)s;
    while (depth[v] == NULLV) {
      if (sp >= N) {
        free(stack);
        return -1;
      }
      stack[sp++] = v;
      uint32_t p  = parents[v];
      if (p == NULLV || p >= N) {
        free(stack);
        return -1;
      }
      v = p;
    }
    uint32_t d = depth[v];
    while (sp) {
      uint32_t w = stack[--sp];
      depth[w]   = ++d;
    }
  }
  free(stack);
  return 0;
}

/* BFSVerifier checks (bfs.hpp:66-97): root is its own parent at depth 0;
 * every reached u has parents[u] in in[u] at depth[u]-1; reachability of
 * parents matches reachability of depths.  Returns 1 if all hold. */
int nwgport_verify(const uint64_t* out_off, const uint32_t* out_col, const uint64_t* in_off, const uint32_t* in_col,
                   uint64_t N, uint32_t root, const uint32_t* parents) {
  if (!in_off) {
    in_off = out_off;
    in_col = out_col;
  }
  uint32_t* depth = (uint32_t*)malloc(sizeof(uint32_t) * (N ? N : 1));
  if (!depth) return -2;
  nwgport_bfs_depths(out_off, out_col, N, root, depth);
  int ok = 1;
  for (uint64_t u = 0; u < N && ok; ++u) {
    if (depth[u] != NULLV && parents[u] != NULLV) {
      if (u == root) {
        ok = (parents[u] == u && depth[u] == 0);
        continue;
      }
      int found = 0;
      for (uint64_t e = in_off[u]; e < in_off[u + 1]; ++e) {
        if (in_col[e] == parents[u]) {
          if (depth[in_col[e]] != depth[u] - 1) ok = 0;
          found = 1;
          break;
        }
      }
      if (!found) ok = 0;
    } else if (depth[u] != parents[u]) {
      ok = 0;
    }
  }
  free(depth);
  return ok;
}

/* uint8 depths for k sources, row-major [k][N]; 255 = unreached.  Returns
 * the maximum finite depth seen, or -3 if some depth is >= 255 (does not fit
 * the uint8 encoding). */
int64_t nwgport_msbfs_depths(const uint64_t* off, const uint32_t* col, uint64_t N, const uint32_t* roots, uint32_t k,
                             uint8_t* depths) {
  uint32_t* d = (uint32_t*)malloc(sizeof(uint32_t) * (N ? N : 1));
  if (!d) return -2;
  int64_t maxd = 0;
  for (uint32_t s = 0; s < k; ++s) {
    if (nwgport_bfs_depths(off, col, N, roots[s], d) < 0) {
      free(d);
      return -1;
    }
    uint8_t* row = depths + (uint64_t)s * N;
    for (uint64_t v = 0; v < N; ++v) {
      if (d[v] == NULLV) {
        row[v] = 255;
      } else if (d[v] >= 255) {
        free(d);
        return -3;
      } else {
        row[v] = (uint8_t)d[v];
        if (d[v] > maxd) maxd = d[v];
      }
    }
  }
  free(d);
  return maxd;
}


/* Approximate betweenness centrality, BCVerifier's own computation
 * (betweenness_centrality.hpp:63-115).  scores: n floats.  Returns 0, or -2
 * when out of memory. */
int64_t nwgport_bc(const uint64_t* off, const uint32_t* col, uint64_t N, const uint32_t* sources, uint32_t k,
                   int normalize, float* scores) {
  int32_t*  depth = (int32_t*)malloc(sizeof(int32_t) * (N ? N : 1));
  double*   pc    = (double*)malloc(sizeof(double) * (N + 1));
  float*    delta = (float*)malloc(sizeof(float) * (N ? N : 1));
  uint32_t* order = (uint32_t*)malloc(sizeof(uint32_t) * (N ? N : 1));
  uint64_t* lvl   = (uint64_t*)malloc(sizeof(uint64_t) * (N + 2));
  if (!depth || !pc || !delta || !order || !lvl) {
    free(depth), free(pc), free(delta), free(order), free(lvl);
    return -2;
  }
  for (uint64_t i = 0; i < N; ++i) scores[i] = 0.0f;
  for (uint32_t si = 0; si < k; ++si) {
    const uint32_t s = sources[si];
    for (uint64_t i = 0; i < N; ++i) {
      depth[i] = -1;
      pc[i]    = 0.0;
      delta[i] = 0.0f;
    }
    depth[s] = 0;
    pc[s]    = 1.0;
    uint64_t head = 0, tail = 0;
    order[tail++] = s;
    /* forward: BFS order with path counts (:66-83) */
    while (head < tail) {
      const uint32_t u = order[head++];
      for (uint64_t e = off[u]; e < off[u + 1]; ++e) {
        const uint32_t v = col[e];
        if (depth[v] == -1) {
          depth[v]      = depth[u] + 1;
          order[tail++] = v;
        }
        if (depth[v] == depth[u] + 1) pc[v] += pc[u];
      }
    }
    /* levels in BFS order are contiguous: lvl[d] = first index of depth d */
    uint64_t nlev = 0;
    for (uint64_t i = 0; i < tail; ++i)
      if (i == 0 || depth[order[i]] != depth[order[i - 1]]) lvl[nlev++] = i;
    lvl[nlev] = tail;
    /* backward, deepest level first (:96-107); within a level the vertices
     * are independent, so their order does not change any value */
    for (int64_t d = (int64_t)nlev - 1; d >= 0; --d) {
      for (uint64_t i = lvl[d]; i < lvl[d + 1]; ++i) {
        const uint32_t u = order[i];
        for (uint64_t e = off[u]; e < off[u + 1]; ++e) {
          const uint32_t v = col[e];
          if (depth[v] == depth[u] + 1) delta[u] += pc[u] / pc[v] * (1 + delta[v]);
        }
        scores[u] += delta[u];
      }
    }
  }
  if (normalize && N) {
    float big = scores[0];
    for (uint64_t i = 1; i < N; ++i)
      if (scores[i] > big) big = scores[i];
    for (uint64_t i = 0; i < N; ++i) scores[i] = scores[i] / big;
  }
  free(depth), free(pc), free(delta), free(order), free(lvl);
  return 0;
}
