/*
 * CPU oracle for the exact-clustering hot path: a plain-C restatement of the
 * reference's (shangar21/cuhc) FP32 arithmetic, used ONLY as the checker by
 * tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg. The product
 * (cuhc_b200/libcuhc.so) never links or calls it.
 *
 * Parity pins (tests/test_oracle.py, tests/test_gpu_parity.py):
 *   - condensed trees against the reference's own cuhc_condense_tree (built
 *     from its sources into oracle/_ref, runs on the CPU here);
 *   - single-linkage trees against scipy.cluster.hierarchy.linkage, the
 *     reference's own test oracle (tests/test_mst.py:18-30 contract);
 *   - core distances against a float64 NumPy sort (tests/test_hdbscan.py:150);
 *   - on a GPU box: bit-for-bit against the reference build run with spatial
 *     pruning off (its tie order is the original point index, as here), and
 *     against committed fixtures made that way (tests/golden/).
 *
 * Arithmetic rules followed exactly (compile with -ffp-contract=off so the
 * compiler fuses nothing on its own):
 *   - per pair, features folded in order 0..d-1 (distances.cuh:21-83):
 *       sqeuclidean: acc = fmaf(a - b, a - b, acc); euclidean adds sqrtf;
 *       manhattan: acc + fabsf(a - b); chebyshev: fmaxf(acc, fabsf(a - b));
 *       cosine: three fmaf accumulators, 1 - dot / sqrtf(|a|^2 * |b|^2),
 *               1 for a zero vector;
 *       minkowski: powf per feature (the reference's device code uses a fast
 *               exp2/log2 form, so minkowski is tolerance-level only).
 *   - argmin keys are (weight bits << 32 | index), weights clamped at 0
 *     (reductions.cuh:64-69), ties to the lower index (reductions.cuh:19-21);
 *   - mutual reachability = fmaxf(fmaxf(core_i, core_j), d or d / alpha)
 *     (hdbscan.cuh:342-351);
 *   - the MST is the unique one under the edge order (weight, smaller
 *     endpoint, larger endpoint) (mst.cuh:41-48). Prim's algorithm with that
 *     total order finds the same tree as the reference's Borůvka rounds.
 *   - single-linkage tree: edges sorted by that order, union-find assigns
 *     scipy ids (mst.cuh:204-235);
 *   - core distance: the k-th smallest distance of a row, the point itself
 *     counted as 0, others clamped at 0 (hdbscan.cuh:205-212, 76-79);
 *   - condensed tree: breadth-first walk from the root with sklearn 1.9's
 *     relabelling rules and row order (hdbscan.cuh:398-483).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

enum { M_EUCLIDEAN = 0, M_SQEUCLIDEAN = 1, M_MANHATTAN = 2, M_CHEBYSHEV = 3, M_MINKOWSKI = 4,
       M_COSINE = 5 };
enum { ERR_METRIC = -1, ERR_SHAPE = -2, ERR_DISCONNECTED = -5, ERR_NONFINITE = -6 };

static int num_threads_setting = 0; /* 0 = OpenMP default */

void orc_set_threads(int threads) { num_threads_setting = threads; }

int orc_get_threads(void) {
#ifdef _OPENMP
  return num_threads_setting > 0 ? num_threads_setting : omp_get_max_threads();
#else
  return 1;
#endif
}

/* Distance between two rows of length d, in the reference's per-metric order. */
static inline float metric_distance(const float *x, const float *y, int d, int metric, float p) {
  switch (metric) {
  case M_EUCLIDEAN:
  case M_SQEUCLIDEAN: {
    float acc = 0.0f;
    for (int k = 0; k < d; ++k) {
      const float diff = x[k] - y[k];
      acc = fmaf(diff, diff, acc);
    }
    return metric == M_EUCLIDEAN ? sqrtf(acc) : acc;
  }
  case M_MANHATTAN: {
    float acc = 0.0f;
    for (int k = 0; k < d; ++k)
      acc = acc + fabsf(x[k] - y[k]);
    return acc;
  }
  case M_CHEBYSHEV: {
    float acc = 0.0f;
    for (int k = 0; k < d; ++k)
      acc = fmaxf(acc, fabsf(x[k] - y[k]));
    return acc;
  }
  case M_MINKOWSKI: {
    float acc = 0.0f;
    for (int k = 0; k < d; ++k)
      acc = acc + powf(fabsf(x[k] - y[k]), p);
    return powf(acc, 1.0f / p);
  }
  case M_COSINE: {
    float dot = 0.0f, xx = 0.0f, yy = 0.0f;
    for (int k = 0; k < d; ++k) {
      dot = fmaf(x[k], y[k], dot);
      xx = fmaf(x[k], x[k], xx);
      yy = fmaf(y[k], y[k], yy);
    }
    const float denom = sqrtf(xx * yy);
    return denom > 0.0f ? 1.0f - dot / denom : 1.0f;
  }
  }
  return NAN;
}

static int valid_metric(int metric) { return metric >= M_EUCLIDEAN && metric <= M_COSINE; }

/* Edge weight of (i, j): the distance, or mutual reachability if core != NULL. */
static inline float edge_weight(const float *X, int d, int metric, float p, const float *core,
                                float alpha, int i, int j) {
  const float dist = metric_distance(X + (size_t)i * d, X + (size_t)j * d, d, metric, p);
  if (!core)
    return dist;
  return fmaxf(fmaxf(core[i], core[j]), alpha == 1.0f ? dist : dist / alpha);
}

static inline uint64_t pack_key(float w, int index) {
  const float clamped = w > 0.0f ? w : 0.0f;
  uint32_t bits;
  memcpy(&bits, &clamped, 4);
  return ((uint64_t)bits << 32) | (uint32_t)index;
}

/* distances[i][j] = metric(A[i], B[j]); B == NULL means B = A. */
int orc_pairwise(const float *A, int nA, const float *B, int nB, int d, int metric, float p,
                 float *out) {
  if (nA <= 0 || nB <= 0 || d <= 0)
    return ERR_SHAPE;
  if (!valid_metric(metric))
    return ERR_METRIC;
  if (!B)
    B = A;
#pragma omp parallel for schedule(static) num_threads(orc_get_threads())
  for (int i = 0; i < nA; ++i)
    for (int j = 0; j < nB; ++j)
      out[(size_t)i * nB + j] = metric_distance(A + (size_t)i * d, B + (size_t)j * d, d, metric, p);
  return 0;
}

/* Inserts v into the ascending list[0..k) if it beats the k-th. */
static inline void insert_sorted(float *list, int k, float v) {
  if (!(v < list[k - 1]))
    return;
  int pos = k - 1;
  while (pos > 0 && list[pos - 1] > v) {
    list[pos] = list[pos - 1];
    --pos;
  }
  list[pos] = v;
}

/* core[i] for rows [rowBegin, rowEnd): k-th smallest distance, self = 0. */
int orc_core_distances_rows(const float *X, int n, int d, int metric, float p, int k,
                            int rowBegin, int rowEnd, float *core) {
  if (n <= 0 || d <= 0 || k < 1 || k > n || rowBegin < 0 || rowEnd > n)
    return ERR_SHAPE;
  if (!valid_metric(metric))
    return ERR_METRIC;
#pragma omp parallel num_threads(orc_get_threads())
  {
    float *list = (float *)malloc((size_t)k * sizeof(float));
#pragma omp for schedule(dynamic, 16)
    for (int i = rowBegin; i < rowEnd; ++i) {
      for (int t = 0; t < k; ++t)
        list[t] = INFINITY;
      for (int j = 0; j < n; ++j) {
        float v = j == i ? 0.0f
                         : metric_distance(X + (size_t)i * d, X + (size_t)j * d, d, metric, p);
        v = j == i ? 0.0f : fmaxf(v, 0.0f);
        insert_sorted(list, k, v);
      }
      core[i - rowBegin] = list[k - 1];
    }
    free(list);
  }
  return 0;
}

int orc_core_distances(const float *X, int n, int d, int metric, float p, int k, float *core) {
  return orc_core_distances_rows(X, n, d, metric, p, k, 0, n, core);
}

/* One nearest-other-component pass, unpruned: nearest[i] = packed (weight,
 * j) minimum over j with component[j] != component[i], ties to the lower j;
 * ~0 when there is none (distance_matrix.cuh:213-271). */
int orc_nearest_other_component(const float *X, int n, int d, int metric, float p,
                                const float *core, float alpha, const int *component,
                                uint64_t *nearest) {
  if (n <= 0 || d <= 0)
    return ERR_SHAPE;
  if (!valid_metric(metric))
    return ERR_METRIC;
#pragma omp parallel for schedule(dynamic, 16) num_threads(orc_get_threads())
  for (int i = 0; i < n; ++i) {
    uint64_t best = ~0ull;
    for (int j = 0; j < n; ++j) {
      if (component[j] == component[i])
        continue;
      const float w = edge_weight(X, d, metric, p, core, alpha, i, j);
      if (w != w)
        continue;
      const uint64_t key = pack_key(w, j);
      if (key < best)
        best = key;
    }
    nearest[i] = best;
  }
  return 0;
}

/* Lexicographic (w, u, v) comparison, weights compared as floats. */
static inline int edge_less(float wa, int ua, int va, float wb, int ub, int vb) {
  if (wa != wb)
    return wa < wb;
  if (ua != ub)
    return ua < ub;
  return va < vb;
}

/* Prim's algorithm under the total order (weight, min endpoint, max
 * endpoint): the unique MST that the reference's Borůvka rounds produce.
 * Edges are written in the order Prim adds them. core != NULL selects mutual
 * reachability weights. Returns 0, or ERR_DISCONNECTED if some point has no
 * finite edge to the rest. */
int orc_mst(const float *X, int n, int d, int metric, float p, const float *core, float alpha,
            int *edgeU, int *edgeV, float *edgeW) {
  if (n <= 0 || d <= 0)
    return ERR_SHAPE;
  if (!valid_metric(metric))
    return ERR_METRIC;
  if (n == 1)
    return 0;
  float *keyW = (float *)malloc((size_t)n * sizeof(float));
  int *keyU = (int *)malloc((size_t)n * sizeof(int));
  int *keyV = (int *)malloc((size_t)n * sizeof(int));
  char *inTree = (char *)calloc((size_t)n, 1);
  const int threads = orc_get_threads();
  for (int v = 0; v < n; ++v) {
    keyW[v] = INFINITY;
    keyU[v] = keyV[v] = -1;
  }
  int status = 0;
  int added = 0; /* vertex just added to the tree */
  inTree[0] = 1;
  for (int step = 0; step < n - 1; ++step) {
    int bestVertex = -1;
#pragma omp parallel num_threads(threads)
    {
      int localBest = -1;
#pragma omp for schedule(static)
      for (int v = 0; v < n; ++v) {
        if (inTree[v])
          continue;
        const float w = edge_weight(X, d, metric, p, core, alpha, added, v);
        const int u = added < v ? added : v, vv = added < v ? v : added;
        if (w == w && (keyU[v] < 0 || edge_less(w, u, vv, keyW[v], keyU[v], keyV[v]))) {
          keyW[v] = w;
          keyU[v] = u;
          keyV[v] = vv;
        }
        if (keyU[v] >= 0 &&
            (localBest < 0 || edge_less(keyW[v], keyU[v], keyV[v], keyW[localBest],
                                        keyU[localBest], keyV[localBest])))
          localBest = v;
      }
#pragma omp critical
      {
        if (localBest >= 0 &&
            (bestVertex < 0 || edge_less(keyW[localBest], keyU[localBest], keyV[localBest],
                                         keyW[bestVertex], keyU[bestVertex], keyV[bestVertex])))
          bestVertex = localBest;
      }
    }
    if (bestVertex < 0 || !isfinite(keyW[bestVertex])) {
      status = ERR_DISCONNECTED;
      break;
    }
    edgeU[step] = keyU[bestVertex];
    edgeV[step] = keyV[bestVertex];
    edgeW[step] = keyW[bestVertex];
    inTree[bestVertex] = 1;
    added = bestVertex;
  }
  free(keyW);
  free(keyU);
  free(keyV);
  free(inTree);
  return status;
}

/* ---- merge tree from MST edges ------------------------------------------ */

typedef struct {
  int u, v;
  float w;
} Edge;

static int cmp_edge(const void *a, const void *b) {
  const Edge *x = (const Edge *)a, *y = (const Edge *)b;
  if (edge_less(x->w, x->u, x->v, y->w, y->u, y->v))
    return -1;
  if (edge_less(y->w, y->u, y->v, x->w, x->u, x->v))
    return 1;
  return 0;
}

static int uf_find(int *parent, int x) {
  while (parent[x] != x) {
    parent[x] = parent[parent[x]];
    x = parent[x];
  }
  return x;
}

/* Z ((n-1) x 4, scipy format) from merges already in tree order: union-find
 * names each merged pair by its current cluster ids (mst.cuh:204-228). */
static void tree_from_ordered(const Edge *edges, int n, double *Z) {
  int *parent = (int *)malloc((size_t)n * sizeof(int));
  int *size = (int *)malloc((size_t)n * sizeof(int));
  int *rank = (int *)calloc((size_t)n, sizeof(int));
  int *id = (int *)malloc((size_t)n * sizeof(int));
  for (int i = 0; i < n; ++i) {
    parent[i] = i;
    size[i] = 1;
    id[i] = i;
  }
  for (int s = 0; s < n - 1; ++s) {
    const int ru = uf_find(parent, edges[s].u), rv = uf_find(parent, edges[s].v);
    const int a = id[ru], b = id[rv];
    const int merged = size[ru] + size[rv];
    Z[(size_t)s * 4 + 0] = a < b ? a : b;
    Z[(size_t)s * 4 + 1] = a < b ? b : a;
    Z[(size_t)s * 4 + 2] = edges[s].w;
    Z[(size_t)s * 4 + 3] = merged;
    /* Any root choice gives the same ids; union by size keeps paths short. */
    int root = ru, child = rv;
    if (size[ru] < size[rv]) {
      root = rv;
      child = ru;
    }
    parent[child] = root;
    size[root] = merged;
    id[root] = n + s;
  }
  free(parent);
  free(size);
  free(rank);
  free(id);
}

/* Single-linkage Z from n-1 MST edges (sorted here by the edge order). */
void orc_tree_from_mst(const int *edgeU, const int *edgeV, const float *edgeW, int n, double *Z) {
  if (n < 2)
    return;
  Edge *edges = (Edge *)malloc((size_t)(n - 1) * sizeof(Edge));
  for (int s = 0; s < n - 1; ++s) {
    const int u = edgeU[s], v = edgeV[s];
    edges[s].u = u < v ? u : v;
    edges[s].v = u < v ? v : u;
    edges[s].w = edgeW[s];
  }
  qsort(edges, (size_t)(n - 1), sizeof(Edge), cmp_edge);
  tree_from_ordered(edges, n, Z);
  free(edges);
}

/* Full single-linkage tree of the points (cuhc_linkage, algorithm "mst"). */
int orc_single_linkage(const float *X, int n, int d, int metric, float p, double *Z) {
  if (n <= 0 || d <= 0)
    return ERR_SHAPE;
  if (n == 1)
    return 0;
  int *u = (int *)malloc((size_t)(n - 1) * sizeof(int));
  int *v = (int *)malloc((size_t)(n - 1) * sizeof(int));
  float *w = (float *)malloc((size_t)(n - 1) * sizeof(float));
  int status = orc_mst(X, n, d, metric, p, NULL, 1.0f, u, v, w);
  if (status == 0)
    orc_tree_from_mst(u, v, w, n, Z);
  free(u);
  free(v);
  free(w);
  return status;
}

/* HDBSCAN's single-linkage tree of mutual reachability plus core distances
 * (cuhc_hdbscan_tree). core may be NULL. */
int orc_hdbscan_tree(const float *X, int n, int d, int metric, float p, int minSamples,
                     float alpha, double *Z, float *coreOut) {
  if (n <= 0 || d <= 0 || minSamples < 1 || minSamples > n)
    return ERR_SHAPE;
  float *core = (float *)malloc((size_t)n * sizeof(float));
  int status = orc_core_distances(X, n, d, metric, p, minSamples, core);
  if (status == 0 && n > 1) {
    int *u = (int *)malloc((size_t)(n - 1) * sizeof(int));
    int *v = (int *)malloc((size_t)(n - 1) * sizeof(int));
    float *w = (float *)malloc((size_t)(n - 1) * sizeof(float));
    status = orc_mst(X, n, d, metric, p, core, alpha, u, v, w);
    if (status == 0)
      orc_tree_from_mst(u, v, w, n, Z);
    free(u);
    free(v);
    free(w);
  }
  if (status == 0 && coreOut)
    memcpy(coreOut, core, (size_t)n * sizeof(float));
  free(core);
  return status;
}

/* ---- condensed tree ------------------------------------------------------ */

/* Breadth-first nodes below `from` (children left then right), appended to
 * out[*count...]. Uses queue as scratch (room for 2n-1 nodes). */
static void bfs_nodes(const double *Z, long long n, long long from, long long *queue,
                      long long *out, long long *count) {
  long long head = 0, tail = 0;
  queue[tail++] = from;
  while (head < tail) {
    const long long node = queue[head++];
    out[(*count)++] = node;
    if (node >= n) {
      queue[tail++] = (long long)Z[(node - n) * 4 + 0];
      queue[tail++] = (long long)Z[(node - n) * 4 + 1];
    }
  }
}

/* sklearn 1.9's condensing of the (n-1) x 4 tree; rows in its order
 * (hdbscan.cuh:398-483 follows the same rules). Returns the row count, or
 * -(rows needed) if capacity is too small. */
long long orc_condense_tree(const double *Z, long long n, long long minClusterSize,
                            long long capacity, long long *parentOut, long long *childOut,
                            double *lambdaOut, long long *sizeOut) {
  if (n < 2)
    return 0;
  const long long root = 2 * (n - 1);
  long long *order = (long long *)malloc((size_t)(root + 1) * sizeof(long long));
  long long *queue = (long long *)malloc((size_t)(root + 1) * sizeof(long long));
  long long *sub = (long long *)malloc((size_t)(root + 1) * sizeof(long long));
  long long *relabel = (long long *)calloc((size_t)(root + 1), sizeof(long long));
  char *ignore = (char *)calloc((size_t)(root + 1), 1);
  long long numOrder = 0;
  bfs_nodes(Z, n, root, queue, order, &numOrder);
  relabel[root] = n;
  long long nextLabel = n + 1, rows = 0;

#define EMIT(P, C, L, S)                                                                           \
  do {                                                                                             \
    if (rows < capacity) {                                                                         \
      parentOut[rows] = (P);                                                                       \
      childOut[rows] = (C);                                                                        \
      lambdaOut[rows] = (L);                                                                       \
      sizeOut[rows] = (S);                                                                         \
    }                                                                                              \
    ++rows;                                                                                        \
  } while (0)

  for (long long t = 0; t < numOrder; ++t) {
    const long long node = order[t];
    if (ignore[node] || node < n)
      continue;
    const double *row = Z + (node - n) * 4;
    const long long left = (long long)row[0], right = (long long)row[1];
    const double dist = row[2];
    const double lambda = dist > 0.0 ? 1.0 / dist : INFINITY;
    const long long leftCount = left >= n ? (long long)Z[(left - n) * 4 + 3] : 1;
    const long long rightCount = right >= n ? (long long)Z[(right - n) * 4 + 3] : 1;
    const int leftBig = leftCount >= minClusterSize, rightBig = rightCount >= minClusterSize;
    if (leftBig && rightBig) {
      relabel[left] = nextLabel++;
      EMIT(relabel[node], relabel[left], lambda, leftCount);
      relabel[right] = nextLabel++;
      EMIT(relabel[node], relabel[right], lambda, rightCount);
      continue;
    }
    /* Sides that are too small drop out point by point, in BFS order. */
    for (int side = 0; side < 2; ++side) {
      const long long child = side == 0 ? left : right;
      const int big = side == 0 ? leftBig : rightBig;
      if (big) {
        relabel[child] = relabel[node];
        continue;
      }
      long long count = 0;
      bfs_nodes(Z, n, child, queue, sub, &count);
      for (long long s = 0; s < count; ++s) {
        if (sub[s] < n)
          EMIT(relabel[node], sub[s], lambda, 1);
        ignore[sub[s]] = 1;
      }
    }
  }
#undef EMIT
  free(order);
  free(queue);
  free(sub);
  free(relabel);
  free(ignore);
  return rows <= capacity ? rows : -rows;
}
