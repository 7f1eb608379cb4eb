/*
 * cuhc.h — C ABI of libcuhc.so (cuhc_b200), the drop-in boundary of the
 * exact-clustering hot path of shangar21/cuhc.
 *
 * The first eight functions replace the reference's ctypes boundary one for
 * one: same symbol names, signatures, argument meaning, id tables and status
 * codes (reference src/capi.cu, bound by its python/cuhc/_lib.py:19-91). A
 * ctypes caller of the reference library can load this one instead.
 *
 * Conventions (as in the reference):
 *   - every pointer is HOST memory owned by the caller, except the *_device
 *     additions, whose point arrays are DEVICE memory on the current device;
 *   - points are row-major float32 (numPoints x numFeatures);
 *   - calls are synchronous; device memory comes from a stream-ordered pool;
 *   - status: 0 success, a positive cudaError_t, or a negative code below.
 *
 * Id tables:
 *   metric     euclidean 0, sqeuclidean 1, manhattan 2, chebyshev 3,
 *              minkowski 4 (order p), cosine 5         (reference capi.cu:17-24)
 *   linkage    single 0, complete 1, average 2, ward 3 (reference linkage.cuh:31)
 *   algorithm  dense 0, mst 1, nn_chain 2, rnn 3       (reference capi.cu:33-38)
 *   coreMethod auto 0, fused 1, radix 2                (reference hdbscan.cuh:324)
 *   pruning    auto 0, always 1, never 2               (reference spatial.cuh:354)
 */
#ifndef CUHC_B200_CUHC_H
#define CUHC_B200_CUHC_H

#ifdef __cplusplus
extern "C" {
#endif

/* Negative status codes; -1..-6 are the reference's (capi.cu:26-30, mst.cuh:80-81). */
#define CUHC_ERROR_INVALID_METRIC (-1)
#define CUHC_ERROR_INVALID_SHAPE (-2)
#define CUHC_ERROR_INVALID_LINKAGE (-3)
#define CUHC_ERROR_INVALID_ALGORITHM (-4)
#define CUHC_ERROR_DISCONNECTED (-5)
#define CUHC_ERROR_NON_FINITE (-6)
/* Additions: a bounded device wait ran out; a size beyond an entry point's limit. */
#define CUHC_ERROR_TIMEOUT (-7)
#define CUHC_ERROR_TOO_LARGE (-8)

/* distances (numPointsA x numPointsB, row-major) = metric(A[i], B[j]);
 * pointsB == NULL means B = A.
 * Replaces reference capi.cu:138-173 (cuhc_pairwise_distances). */
int cuhc_pairwise_distances(const float *pointsA, int numPointsA, const float *pointsB,
                            int numPointsB, int numFeatures, int metricId, float metricParam,
                            float *distances);

/* Full merge tree in scipy's linkage format: tree receives (numPoints - 1) x 4
 * doubles {id1, id2, height, size}. mst needs single linkage; rnn and
 * nn_chain need ward with euclidean; dense builds any linkage.
 * Replaces reference capi.cu:179-257 (cuhc_linkage). */
int cuhc_linkage(const float *points, int numPoints, int numFeatures, int metricId,
                 float metricParam, int linkageId, int algorithmId, double *tree);

/* Ward through RNN rounds with explicit hand-over settings (test hook).
 * Replaces reference capi.cu:261-279 (cuhc_ward_rnn_with_options). */
int cuhc_ward_rnn_with_options(const float *points, int numPoints, int numFeatures,
                               float minProgress, int denseBelow, int allowDense, double *tree);

/* HDBSCAN's single-linkage tree of mutual reachability,
 * max(core_i, core_j, d(i, j) / alpha); core (may be NULL) receives the core
 * distances (distance to the minSamples-th nearest point, itself first).
 * Replaces reference capi.cu:285-309 (cuhc_hdbscan_tree). */
int cuhc_hdbscan_tree(const float *points, int numPoints, int numFeatures, int metricId,
                      float metricParam, int minSamples, float alpha, int coreMethod,
                      double *tree, float *core);

/* HDBSCAN's condensed tree of a (numPoints - 1) x 4 tree: up to capacity rows
 * into the four arrays; returns the row count, or -(rows needed).
 * Replaces reference capi.cu:314-327 (cuhc_condense_tree). */
long long cuhc_condense_tree(const double *tree, long long numPoints, long long minClusterSize,
                             long long capacity, long long *parent, long long *child,
                             double *lambda, long long *size);

/* Spatial pruning of the matrix-free paths; results never change.
 * Replaces reference capi.cu:332-337 (cuhc_set_pruning). */
int cuhc_set_pruning(int mode);

/* Tiles computed and tiles in total by the passes since the last call; resets.
 * Replaces reference capi.cu:341-345 (cuhc_prune_stats). */
void cuhc_prune_stats(unsigned long long *computed, unsigned long long *total);

/* Message for a status code.
 * Replaces reference capi.cu:347-364 (cuhc_error_string). */
const char *cuhc_error_string(int code);

/* ---- additions (no counterpart in the reference) ------------------------ */

/* cuhc_linkage with the points already in device memory (current device). */
int cuhc_linkage_device(const float *devicePoints, int numPoints, int numFeatures, int metricId,
                        float metricParam, int linkageId, int algorithmId, double *tree);

/* cuhc_hdbscan_tree with the points already in device memory. */
int cuhc_hdbscan_tree_device(const float *devicePoints, int numPoints, int numFeatures,
                             int metricId, float metricParam, int minSamples, float alpha,
                             int coreMethod, double *tree, float *core);

/* cuhc_pairwise_distances with A, B (NULL means B = A, then numPointsB ==
 * numPointsA) and the numPointsA x numPointsB output in device memory of the
 * current device; synchronous. */
int cuhc_pairwise_distances_device(const float *devicePointsA, int numPointsA,
                                   const float *devicePointsB, int numPointsB, int numFeatures,
                                   int metricId, float metricParam, float *deviceDistances);

/* HDBSCAN labels (-1 = noise) and membership probabilities of a (n-1) x 4
 * single-linkage tree (HOST memory), scikit-learn 1.9 extraction semantics.
 * method: 0 excess of mass, 1 leaf; maxClusterSize <= 0 means no limit.
 * Replaces the NumPy extraction of reference python/cuhc/_hdbscan.py:148-350
 * (no counterpart in its C ABI). */
int cuhc_hdbscan_labels(const double *tree, long long n, long long minClusterSize, int method,
                        int allowSingleCluster, double epsilon, long long maxClusterSize,
                        long long *labels, double *probabilities);

/* Trees of many instances in one batched solve (no counterpart in the
 * reference; its callers make one cuhc_linkage / cuhc_hdbscan_tree call per
 * instance). Instance i is rows [offsets[i], offsets[i+1]) of the HOST array
 * points (numFeatures columns, float32); offsets has count + 1 entries,
 * offsets[0] = 0, every instance at least one row. minSamples[i] = 0 gives
 * its single-linkage tree, k >= 1 (k <= 256 and <= its rows) HDBSCAN's tree of
 * mutual reachability with min_samples k, alpha 1. Instance i's tree,
 * (n_i - 1) x 4 doubles, starts at row offsets[i] - i of `trees`; core (may
 * be NULL) receives every point's core distance (0 for single linkage). Each
 * tree is bit-identical to the per-instance call's. All instances share one
 * k-d forest, one k-NN pass and one Borůvka solve whose rounds after the
 * first replay as a CUDA graph. */
int cuhc_trees_batched(const float *points, const long long *offsets, int count, int numFeatures,
                       int metricId, float metricParam, const int *minSamples, double *trees,
                       float *core);

/* cuhc_trees_batched with the points already in device memory. */
int cuhc_trees_batched_device(const float *devicePoints, const long long *offsets, int count,
                              int numFeatures, int metricId, float metricParam,
                              const int *minSamples, double *trees, float *core);

/* ---- learned radius proposal (no counterpart in the reference) ----------
 * Single-linkage Borůvka rounds over 16 features can cap each row's search at
 * a radius proposed by a 19 -> 64 -> 64 -> 1 BF16 MLP (5,505 parameters:
 * W1[19][64], b1[64], W2[64][64], b2[64], w3[64], b3), certify the rows whose
 * best edge lies inside it and search the rest again: trees never change. */

/* Loads the model (HOST params) with its calibration offset (radius =
 * exp(prediction + offset)); params NULL switches the proposal off. */
int cuhc_set_radius_model(const float *params, float offset);
/* Since the last call (first `count` of: rows proposed, rows certified,
 * tiles of the capped passes, tiles of the fallback passes). */
int cuhc_radius_stats(unsigned long long *out, int count);
/* The pipeline shape (ring slots, copy lead) that the shape tuner chose for
 * the latest screened k-NN pass (0, 0 before any). No counterpart in the
 * reference: the tuner times candidate shapes once per (metric, d, k). */
int cuhc_screen_shape(int *stages, int *lead);
/* Up to maxRowsPerRound random rows per exact single-linkage round of points
 * (HOST, n x 16): features [rows][19], targets (log nearest other-component
 * weight); at most `capacity` rows written, *rows = rows found. */
int cuhc_radius_training_rows(const float *points, int n, int numFeatures, int maxRowsPerRound,
                              unsigned long long seed, float *features, float *targets,
                              long long capacity, long long *rows);
/* The MLP on HOST buffers: forward (x [count][19] -> out), gradient of the
 * mean squared error (and the error), and Adam training in place. */
int cuhc_mlp_forward(const float *params, const float *x, int count, float *out);
int cuhc_mlp_gradient(const float *params, const float *x, const float *y, int count, float *grad,
                      float *loss);
int cuhc_mlp_train(const float *x, const float *y, int count, int epochs, int batch, float lr,
                   unsigned long long seed, float *params, float *losses);

/* Tensor-core screening of the all-pairs passes: 0 auto (on for euclidean and
 * sqeuclidean up to 32 features), 1 on where supported, 2 off. Results never
 * change; returns CUHC_ERROR_INVALID_ALGORITHM for other values. */
int cuhc_set_screen(int mode);

/* Cumulative counters since load: out[0] tiles computed, out[1] tiles in all
 * passes, out[2] passes, out[3] Borůvka rounds (first `count` of them). */
int cuhc_pass_stats(unsigned long long *out, int count);

/* cuhc_pairwise_distances for callers that cannot allocate GPU memory (a
 * host framework owns every device allocation, or an allocation on this path
 * could block or fail). No counterpart in the reference. A, B (NULL means
 * B = A, then numPointsB == numPointsA) and the output are DEVICE memory; the
 * kernel's scratch is a fixed 32 MiB device array inside the library, shared
 * by all calls, so calls that overlap on the GPU race. The work is enqueued
 * on `stream` (NULL: default stream) and not waited for. The first call on a
 * device sets up the array's address; make it before any stream capture.
 * Inputs whose tiled copies exceed the 32 MiB return CUHC_ERROR_TOO_LARGE. */
int cuhc_pairwise_distances_noalloc(const float *devicePointsA, int numPointsA,
                                    const float *devicePointsB, int numPointsB, int numFeatures,
                                    int metricId, float metricParam, float *deviceDistances,
                                    void *stream);

/* Audit of the tensor-core screen (no counterpart in the reference; a test
 * and measurement hook, off by default): with on = 1, every pair of every
 * screened tile is also compared with the reference FP32 squared distance s
 * and an FP64 recomputation. Results never change; audited passes are
 * slower. */
int cuhc_set_screen_audit(int on);

/* Audit results of the current device since the last call, decoded into the
 * first `count` of: pairs audited; pairs whose screened value D' exceeded
 * s + 2^-70 (the screen's guarantee; must be 0); the smallest slack
 * (s - D') / (e (|x|^2 + |y|^2)) with x, y the centred coordinates and e the
 * screen's margin; the largest (s64 - D') / (|x|^2 + |y|^2); the largest
 * s64 - D'; the largest |s - s64| and |s - s64| / s64. NaN where nothing was
 * observed. Resets them. */
int cuhc_screen_audit(double *out, int count);

/* Self-test of the bounded device waits (no counterpart in the reference;
 * the reference's cooperative chain spins without a limit, nn_chain.cuh:84-170).
 * kind 0: the NN-chain kernel's grid barrier over a 4-block cooperative
 * launch; kind 1: the pass kernels' mbarrier wait. missing != 0 leaves one
 * arrival out (a block that returns first; an arrival never made), so every
 * waiter must give up after about limitMicroseconds (1 .. 1,000,000) and the
 * call returns CUHC_ERROR_TIMEOUT with the context still usable; missing == 0
 * must return 0. */
int cuhc_wait_selftest(int kind, int missing, int limitMicroseconds);

/* Number of this library's own kernel launches since load. */
unsigned long long cuhc_launch_count(void);

/* Per-pass CUDA-event timing on the launching stream: on != 0 switches it on. */
int cuhc_set_timing(int on);

/* Per pass kind (0 k-NN pass, 1 nearest-other-component pass, 2 screened
 * nearest pass, 3 screened k-NN pass): device milliseconds, launches and tiles computed since the last
 * call (first `count` kinds); resets them. */
int cuhc_kernel_timing(double *ms, unsigned long long *launches, unsigned long long *tiles,
                       int count);

/* Screened-pass counters since the last call, summed while timing is on
 * (first `count` of): exact FP32 rechecks, row visits that took the exact
 * path, tiles whose components were excluded by indicator slots, tiles
 * masked by component in the epilogue, candidate tiles that no row of their
 * block needed. Resets them. */
int cuhc_screen_counters(unsigned long long *out, int count);

#ifdef __cplusplus
}
#endif

#endif /* CUHC_B200_CUHC_H */
