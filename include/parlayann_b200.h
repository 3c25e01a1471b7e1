/*
 * parlayann_b200.h -- C ABI of the B200 (sm_100a) implementation of
 * ParlayANN's beam search and Vamana build.
 *
 * Every entry point returns an int status (PANN_OK = 0) and records a message
 * for pann_last_error() on failure; none aborts the process. Plain pointers
 * and sizes only. Host-buffer entry points copy inputs in and results out and
 * return when results are in the caller's buffers; *_device entry points take
 * device pointers and a cudaStream_t (passed as void*) and return without
 * synchronising.
 *
 * An index owns the scratch buffers of the searches and the build run on it:
 * calls on one index are made from one host thread at a time. Batch objects
 * (pann_batch_*) own their scratch, so different batches over one index may
 * run from different threads and streams; a server (pann_server_*) takes
 * requests from any thread.
 *
 * Each declaration names the reference interface it replaces
 * (paths relative to the ParlayANN checkout).
 */
#ifndef PARLAYANN_B200_H_
#define PARLAYANN_B200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes; the reference abort()s in these cases
 * (beamSearch.h:51-57,507-511,557-562; graph.h:79-83; index.h:193-199) */
#define PANN_OK 0
#define PANN_EINVAL 1    /* bad argument (k > L, no start point, bad id, ...) */
#define PANN_ENOMEM 2    /* device or host allocation failed */
#define PANN_ETIMEOUT 3  /* a bounded device wait gave up */
#define PANN_EDEVICE 4   /* CUDA error, or no usable sm_100 device */
#define PANN_EOVERFLOW 5 /* a query's seen-set or visited list outgrew every tier */
#define PANN_ESHORT 6    /* a query returned fewer than k results (beamSearch.h:557-562) */

/* element types: uint8_t, int8_t, float (Euclidian_Point<T> / Mips_Point<T>) */
#define PANN_U8 0
#define PANN_I8 1
#define PANN_F32 2
/* distances: Euclidian (euclidian_point.h:45-90) and mips (mips_point.h:44-66) */
#define PANN_L2 0
#define PANN_MIPS 1

typedef struct pann_index pann_index;

/* QueryParams (algorithms/utils/types.h:233-252): k, beamSize, limit,
 * degree_limit, batch_factor. */
typedef struct {
  uint32_t k;
  uint32_t beam;          /* beamSize (L) */
  uint64_t limit;         /* maximum number of visited nodes */
  uint32_t degree_limit;  /* neighbours read per visited node */
  double batch_factor;    /* deferral threshold, fraction of beam; above 1 the reference's
                             set_union can overrun its merge buffer (beamSearch.h:95-96,202-205),
                             while here the buffers hold every deferred candidate */
} pann_query_params;

/* BuildParams fields used by the Vamana build (types.h:155-230). */
typedef struct {
  uint32_t R;             /* max degree */
  uint32_t L;             /* build beam */
  double alpha;
  int32_t num_passes;     /* alpha = 1.0 on all but the last pass (index.h:173-178) */
  double batch_factor;    /* QueryParams.batch_factor of the build searches */
  uint64_t perm_seed;     /* insertion order when perm == NULL */
  int32_t sort_neighbors; /* final per-vertex sort by distance (index.h:180-185) */
} pann_build_params;

/* Per-query counters of stats<T> (stats.h:120-155) plus seen-set diagnostics. */
typedef struct {
  double seconds;          /* whole build, device time */
  double search_seconds;   /* beam search phase (t_beam, index.h:245,275) */
  double prune_seconds;    /* robustPrune of inserted points (inside t_beam) */
  double reverse_seconds;  /* reverse edges: group + append/prune (t_bidirect + t_prune) */
  uint64_t dist_cmps;      /* distance comparisons of searches + prunes */
  uint64_t visited_total;  /* sum of visited-list sizes */
  uint32_t batches;        /* batch_insert rounds over all passes */
  uint32_t flagged;        /* searches where the reference hashset would have grown */
  /* work counters (the build's algorithmic bytes are computed from these) */
  uint64_t search_cmps;      /* distance comparisons of the insertion searches */
  uint64_t prune_candidates; /* candidates assembled for robustPrune (insertions and re-prunes) */
  uint64_t edge_pairs;       /* reverse-edge (neighbour, point) pairs grouped */
  uint64_t reprunes;         /* vertices re-pruned because their reverse edges overflowed R */
  uint64_t inserted;         /* points inserted over all passes */
} pann_build_stats;

/* ---------------------------------------------------------------- index */

/* Create an empty index on the current CUDA device: n points of dimension d,
 * element type dtype (PANN_U8/I8/F32), distance metric (PANN_L2/MIPS), graph
 * max degree R. Replaces PointRange<P>(...) + Graph<uint>(maxDeg, n)
 * (point_range.h:54-117, graph.h:147-149). */
int pann_index_create(pann_index** out, int dtype, int metric, uint64_t n, uint32_t d, uint32_t R);
int pann_index_destroy(pann_index* idx);

/* Load the n x d vectors (dense, row-major) into HBM. on_device != 0 means
 * `vectors` is a device pointer. Replaces PointRange(char* file)
 * (point_range.h:74-117). */
int pann_index_set_points(pann_index* idx, const void* vectors, int on_device);

/* Upload / download the graph in the reference layout: n rows of R+1 uint32,
 * slot 0 = degree (graph.h:138-145,239-247). */
int pann_graph_upload(pann_index* idx, const uint32_t* rows, int on_device);
int pann_graph_download(pann_index* idx, uint32_t* rows);

/* Read / write the reference's graph file: uint32 n, uint32 maxDeg,
 * uint32 deg[n], then the edges (Graph(char*) graph.h:151-208, save graph.h:210-237). */
int pann_graph_load(pann_index* idx, const char* path);
int pann_graph_save(pann_index* idx, const char* path);

/* ---------------------------------------------------------------- search */

/* Beam search for nq queries from the given start points with one set of
 * QueryParams; host buffers. Writes the first k frontier entries (ids,
 * distances) per query, and per-query visited-list size and distance
 * comparisons (stats<T> counters). Any of out_dists / out_visited / out_cmps /
 * out_flags may be NULL. out_flags[i] bit 0 is set where the reference's hashset grows
 * on query i (hashset.h:25-38); those queries are reproduced by an exact
 * emulation of that hashset, so results still equal the reference's. Bit 1
 * is set where a tile search (pann_search_options::parents) stopped early.
 * Replaces qsearchAll / searchAll / beam_search (beamSearch.h:420-445,
 * 492-526, 599-646). */
int pann_search(pann_index* idx, const void* queries, uint32_t nq, const pann_query_params* qp,
                const uint32_t* starts, uint32_t n_start, uint32_t* out_ids, float* out_dists,
                uint32_t* out_visited, uint32_t* out_cmps, uint32_t* out_flags);

/* Same, with every buffer in device memory, on `stream` (a cudaStream_t;
 * 0 is the legacy default stream).
 * Does not synchronise. d_out_flags (may be NULL) receives per-query status
 * bits: 2 = the reference's hashset grows on this query (result reproduced
 * exactly), 1 or 16 = the query's state outgrew every buffer (result invalid),
 * 4 = fewer than k results. starts is a HOST array. Part of the work (the
 * exact emulation of the reference's hashset, beside the first search tier)
 * may run on a stream the index owns; it is ordered after the work already
 * on `stream` and before the rest of this call's work on `stream` by events,
 * so to the caller the call behaves as work on `stream` alone. The queries
 * are taken farthest from the first start point first (results do not
 * depend on the order). Searches on one index share its scratch buffers:
 * device calls on the same index must be ordered on the GPU (one stream, or
 * an event between them); concurrent work uses batch objects
 * (pann_batch_create) or a server (pann_server_create), which own theirs. */
int pann_search_device(pann_index* idx, const void* d_queries, uint32_t nq, const pann_query_params* qp,
                       const uint32_t* starts, uint32_t n_start, uint32_t* d_out_ids, float* d_out_dists,
                       uint32_t* d_out_visited, uint32_t* d_out_cmps, uint32_t* d_out_flags, void* stream);

/* pann_search_device that allocates no device memory. This entry point has
 * no counterpart in the reference. It is for callers that must not call
 * cudaMalloc / cudaFree while they serve queries: cudaFree waits for the whole
 * device to go idle (stalling every other stream on it), a framework's
 * caching allocator may already hold the device's memory, and a latency-bound
 * request path cannot afford an allocation that only its first large batch
 * would trigger.
 *
 * Same arguments, results and status bits as pann_search_device (the same
 * ids, distances, visited and comparison counts). All working memory comes
 * from one statically declared device array of PANN_NOALLOC_SCRATCH_BYTES,
 * which every device that loads this library holds until the process exits;
 * the call makes no cudaMalloc / cudaFree and calls no allocating library
 * routine. A call whose working set does not fit (too many queries, or a
 * beam and degree limit whose seen tables are too large) returns PANN_EINVAL
 * with a message giving the bytes needed; split the batch.
 *  - Every call looks up the array's device address with the index's device
 *    current (the first lookup on a device may load the module that holds
 *    it; make that first call before any stream capture). The address is
 *    not cached, so after a device reset the next call uses the new
 *    context's array. The index's device must be the current device.
 *  - starts is a HOST array copied with cudaMemcpyAsync on `stream`: from
 *    pageable memory the copy is staged before the call returns; from
 *    page-locked memory it is not, so keep the array unchanged until the
 *    stream has reached this call.
 *  - Every call shares the array and finds the previous call's contents in
 *    it; each call clears what must start at zero. Calls that overlap on the
 *    GPU (on different streams, or for different indexes on one device) race
 *    on the array: serialise them (one stream, or an event between).
 *  - The index's own buffers are not used, so it mixes freely with the other
 *    entry points on one index. */
#define PANN_NOALLOC_SCRATCH_BYTES (32u << 20)
int pann_search_device_noalloc(pann_index* idx, const void* d_queries, uint32_t nq, const pann_query_params* qp,
                               const uint32_t* starts, uint32_t n_start, uint32_t* d_out_ids, float* d_out_dists,
                               uint32_t* d_out_visited, uint32_t* d_out_cmps, uint32_t* d_out_flags, void* stream);

/* Beam search returning the reference's full per-query output: the final
 * frontier (<= beam entries, sorted by (distance, id)) and the visited list
 * (sorted by (distance, id)), as filtered_beam_search returns them
 * (beamSearch.h:225-227), plus full_dist_cmps. Host buffers:
 * frontier_ids/frontier_d nq x beam, visited_ids/visited_d nq x visited_cap.
 * A query that visits more than visited_cap nodes fails with PANN_EOVERFLOW.
 * Replaces beam_search / filtered_beam_search (beamSearch.h:33-228,420-445). */
int pann_search_lists(pann_index* idx, const void* queries, uint32_t nq, const pann_query_params* qp,
                      const uint32_t* starts, uint32_t n_start, uint32_t* frontier_ids, float* frontier_d,
                      uint32_t* frontier_n, uint32_t visited_cap, uint32_t* visited_ids, float* visited_d,
                      uint32_t* visited_n, uint32_t* out_cmps);

/* ---------------------------------------------------------------- precision form */

/* Precision of the traversal for float32 indexes. PANN_PREC_F32 is the exact
 * reference search. PANN_PREC_BF16 / PANN_PREC_FP8 score candidates from a
 * low-precision copy of the points (bfloat16; or FP8 E4M3 with one scale per
 * dimension, scale = max |x| / 448) with float32 accumulation, then re-rank the
 * best `rerank` frontier entries (default 4k) with the exact float32 distance,
 * like beam_search_rerank's full-precision pass (beamSearch.h:569-587). The
 * seen-set, visited list and traversal rules are unchanged. */
#define PANN_PREC_F32 0
#define PANN_PREC_BF16 1
#define PANN_PREC_FP8 2

typedef struct {
  int32_t precision; /* PANN_PREC_* */
  uint32_t rerank;   /* candidates re-ranked in float32 (0 = 4k) */
  uint32_t parents;  /* 0: the reference's traversal (one node expanded per step). > 0 (low precision
                        only): the tile search, one CTA per query expanding up to `parents` (<= 4)
                        frontier nodes per step and scoring their new neighbours as one tile staged in
                        shared memory; its own visiting order and recall curve. Status bit 32 marks a
                        query whose seen set filled (it stopped early). */
  uint32_t scorer;   /* tile search only: PANN_SCORER_CUDA scores each staged row on the CUDA cores (one
                        row a thread, float32 FMA); PANN_SCORER_TENSOR scores 128 staged rows at a time
                        on the tensor cores (tcgen05.mma, float32 accumulation in tensor memory; the
                        query split into bfloat16 hi + lo, or three FP8 terms), with the rows' squared
                        norms precomputed by pann_index_set_precision. Rows must be a whole number of
                        32-byte MMA steps (bfloat16: d a multiple of 16; FP8: of 32). */
} pann_search_options;
#define PANN_SCORER_CUDA 0
#define PANN_SCORER_TENSOR 1

/* Distances of given (query, point) pairs: queries nq rows (host), ids nq x m
 * point ids (host), out nq x m (host). PANN_PREC_F32 gives Point::distance
 * exactly (euclidian_point.h:54-90, mips_point.h:44-66: integer sums, or the
 * float32 sequential sum); PANN_PREC_BF16 / PANN_PREC_FP8 give the precision
 * form's approximate scores, the ones its traversal ranks candidates by
 * (pann_index_set_precision first). The reference's counterpart is calling
 * Point::distance on each pair. */
int pann_score(pann_index* idx, const void* queries, uint32_t nq, const uint32_t* ids, uint32_t m, int precision,
               float* out);

/* Build the low-precision copy of the points used by `precision` (kept until
 * the next call; PANN_PREC_F32 frees it). No reference counterpart: the
 * reference's closest feature is its scalar quantization (euclidian_point.h:98-109). */
int pann_index_set_precision(pann_index* idx, int precision);

/* pann_search with options. on_device != 0: every buffer is device memory and
 * the call is asynchronous on `stream` (as pann_search_device); else host
 * buffers and a synchronous call (as pann_search). */
int pann_search_ex(pann_index* idx, const void* queries, uint32_t nq, const pann_query_params* qp,
                   const pann_search_options* opt, const uint32_t* starts, uint32_t n_start, uint32_t* out_ids,
                   float* out_dists, uint32_t* out_visited, uint32_t* out_cmps, uint32_t* out_flags, int on_device,
                   void* stream);

/* ---------------------------------------------------------------- range search */

/* rangeQueryType (types.h:153) */
#define PANN_RANGE_GREEDY 1
#define PANN_RANGE_DOUBLING 2
#define PANN_RANGE_BEAM 3

typedef struct {
  uint32_t beam;                  /* QP.beamSize: the beam search's width (and k) */
  int32_t type;                   /* PANN_RANGE_* */
  double radius;                  /* in Point::distance units: squared L2, or the negated inner product */
  double early_stopping_radius;   /* QP.early_stopping_radius */
  uint32_t early_stopping_count;  /* QP.early_stopping_count; 0 disables early stopping (earlyStopping.h:24-25) */
} pann_range_params;

/* Range search from one start point, as RangeSearch (type GREEDY or BEAM,
 * rangeSearch.h:183-276) and DoubleBeamRangeSearch (type DOUBLING,
 * doublingSearch.h:50-157) compute it on unquantized points: a beam search of
 * width `beam` with early stopping (earlyStopping.h:19-29); its frontier
 * entries within `radius` are the answer, unless all `beam` are within it and
 * the type is GREEDY, in which case greedy_search (rangeSearch.h:21-55)
 * expands from them and its discovery order is the answer (duplicates that
 * the reference's hashset lets through included). Host buffers: answer i is
 * out_ids[out_offsets[i] .. out_offsets[i+1]) (out_offsets has nq + 1
 * entries). If the answers need more than ids_cap ids (or out_ids is NULL
 * and ids_cap 0, to learn the size), out_offsets and the counts are filled,
 * out_ids is not, PANN_EOVERFLOW is returned, and the answers stay on the
 * device for pann_range_fetch. out_visited / out_cmps (may be NULL) get the QueryStats
 * counts; out_flags (may be NULL): bit 0 = the beam's hashset grew, bit 1 =
 * the expansion's hashset grew (both reproduced exactly). */
int pann_range_search(pann_index* idx, const void* queries, uint32_t nq, const pann_range_params* rp,
                      uint32_t start_point, uint64_t* out_offsets, uint32_t* out_ids, uint64_t ids_cap,
                      uint32_t* out_visited, uint32_t* out_cmps, uint32_t* out_flags);

/* The answers of the last pann_range_search (or pann_range_groundtruth) on
 * this index that returned PANN_EOVERFLOW for want of room, into out_ids (ids_cap >= the
 * out_offsets[nq] that call reported), without searching again. The reference
 * sizes each answer vector as it fills (all_neighbors, rangeSearch.h:193,
 * :242-257); a caller with fixed host buffers asks for the size first and
 * fetches the held answers with this. They are held until the next
 * range search or range groundtruth on the index; PANN_EINVAL if none are held. */
int pann_range_fetch(pann_index* idx, uint32_t* out_ids, uint64_t ids_cap);

/* ---------------------------------------------------------------- quantized search */

/* The reference's own mixed-precision search for float indexes: the beam
 * search runs on one-byte scalar-quantized points and the frontier is
 * re-ranked with float distances (beam_search_rerank, beamSearch.h:529-597,
 * as GraphIndex::search_dispatch calls it, python/graph_index.cpp:140-185).
 *
 * pann_index_set_quantized builds the quantized copy. Euclidean indexes: as
 * PointRange<Euclidian_Point<uint8_t>>(Points) does (euclidian_point.h:186-240):
 * slope = 255 / (max - min) over every value with 0 included (all
 * non-negative integers: [0, 255]), offset = round(min * slope), each value
 * round(x * slope) - offset clamped to [0, 255]. Mips indexes: as
 * PointRange<Quantized_Mips_Point<8, true>>(Points) does (mips_point.h:293-499):
 * per point the minimum and maximum value (0 included), the minimum of rank
 * (size_t)(1e-4 n) of the minima and the maximum of rank (size_t)((1 - 1e-4)
 * (n - 1)) of the maxima, bound = max(max, -min), scale = 127 / bound, each
 * value round(x * scale) as int8 (+-127 beyond +-bound); the reference
 * normalises mips points and queries first, which callers of this ABI do
 * themselves. Call it again after pann_index_set_points.
 * pann_index_quant_params returns the slope and offset (mips: the scale and 0). */
int pann_index_set_quantized(pann_index* idx);
int pann_index_quant_params(const pann_index* idx, float* slope, int32_t* offset);

/* Host buffers, float queries (nq x d). The queries are quantized the same
 * way, the search over the quantized points (QueryParams qp, exact as
 * pann_search on a uint8 Euclidean / int8 mips index) keeps min(k * rerank_factor, beam) frontier
 * entries, these are re-scored with the float distance and ordered by
 * (distance, id), and the first k written (out_ids/out_dists nq x k).
 * out_visited / out_cmps (may be NULL) are the quantized search's counts, as
 * QueryStats records them. PANN_ESHORT if a frontier holds fewer than k
 * entries (the reference aborts, beamSearch.h:557-562). */
int pann_search_quantized(pann_index* idx, const void* queries, uint32_t nq, const pann_query_params* qp,
                          double rerank_factor, const uint32_t* starts, uint32_t n_start, uint32_t* out_ids,
                          float* out_dists, uint32_t* out_visited, uint32_t* out_cmps);

/* ---------------------------------------------------------------- batched form */

/* A batch object: a reusable launch sequence for many queries whose k and beam
 * differ per query, with its device buffers allocated once. The reference runs
 * such mixes as one parlay::parallel_for over beam_search calls with
 * different QueryParams (beamSearch.h:492-526); here every run is one
 * persistent, work-stealing launch per tier in which queries are taken
 * longest-beam first, optionally replayed from a CUDA graph captured on the
 * first run. Per query the results equal pann_search's with QueryParams
 * (k[i], beam[i], limit, degree_limit, batch_factor) — exact, bit for bit, on
 * the PANN_PREC_F32 path.
 *
 * bounds->k / bounds->beam are the largest k and beam any run may use (output
 * rows have bounds->k entries; entries past a query's own k are PAD /
 * 0.0f); bounds->limit, degree_limit and batch_factor apply to every query.
 * opt may be NULL (exact float32). */
typedef struct pann_batch pann_batch;

typedef struct {
  int32_t use_graph; /* capture the device launch sequence as a CUDA graph on the first run, replay it after */
  int32_t autotune;  /* time the mappings on the first run and keep the fastest (pann_batch_mapping lists the
                        candidates' knobs: warp per query with the tier-0 seen-table size, warps per block and
                        register budget, or CTA per query; the tile search's rows per round) */
  uint32_t seen_slots;      /* tier-0 seen-table slots (power of two; 0 = automatic) */
  uint32_t warps_per_block; /* tier-0 warps per block (1, 2 or 4; 0 = automatic) */
  int32_t cta_per_query;    /* exact search: 1 runs every query on one block of the exact-emulation kernel
                               (CTA per query) instead of a warp of the first tier; same answers */
} pann_batch_options;

int pann_batch_create(pann_batch** out, pann_index* idx, uint32_t max_queries, const pann_query_params* bounds,
                      const uint32_t* starts, uint32_t n_start, const pann_search_options* opt,
                      const pann_batch_options* bopt);

/* Run nq <= max_queries queries. k and beam are HOST arrays of nq entries
 * (checked: 1 <= k[i] <= beam[i] <= bounds->beam, k[i] <= bounds->k,
 * beam[i] >= n_start). on_device != 0: queries and outputs are device memory
 * and the call is asynchronous on `stream`; else host memory and the call
 * returns when the results are in place. out_ids / out_dists rows have
 * bounds->k entries. out_flags as in pann_search_device (device) or
 * pann_search (host). */
int pann_batch_run(pann_batch* b, const void* queries, uint32_t nq, const uint32_t* k, const uint32_t* beam,
                   uint32_t* out_ids, float* out_dists, uint32_t* out_visited, uint32_t* out_cmps,
                   uint32_t* out_flags, int on_device, void* stream);

/* The launch configuration in use (after autotuning, if any): tier-0 seen
 * slots, warps per block, blocks, and whether a CUDA graph is replayed.
 * Any pointer may be NULL. */
int pann_batch_config(const pann_batch* b, uint32_t* seen_slots, uint32_t* warps_per_block, uint32_t* blocks,
                      int32_t* graph_captured);
/* The mapping the batch runs with (after autotuning, if any): 1 if every query
 * runs on one block of the exact-emulation kernel (CTA per query) instead of a
 * warp of the first tier, the resident blocks per SM the first tier's
 * registers are fitted to (3 or 4), and the tile search's rows staged per
 * round (0 = chosen for occupancy). Any pointer may be NULL. No reference
 * counterpart (the reference runs one thread per query). */
int pann_batch_mapping(const pann_batch* b, uint32_t* cta_per_query, uint32_t* register_blocks, uint32_t* tile_rows);

/* Frees the batch. Device-buffer runs are asynchronous: call this after the
 * last run's stream work has completed (host-buffer runs are synchronous).
 * The index may already have been destroyed. */
int pann_batch_destroy(pann_batch* b);

/* ---------------------------------------------------------------- serving form */

/* A request loop over one resident index (no counterpart in the reference,
 * which searches closed batches: qsearchAll, beamSearch.h:599-646). Requests
 * are submitted from any thread and answered asynchronously: a dispatcher
 * thread keeps up to `inflight` batches on the GPU, each in a slot with a
 * device scratch arena of scratch_bytes, and fills every slot that frees up
 * with the waiting k-NN requests in arrival order while the batch they form
 * fits the arena (admission by scratch memory: a batch needs its queries and
 * outputs, per-query work lists and hand-off records sized by its largest
 * beam, and per-warp seen tables, so requests with small k and beam pack
 * more queries into a slot) and holds at most max_batch_queries queries
 * (continuous batching: requests that arrive while others run join the next
 * slot, and batches overlap on the device). Range requests run on a second
 * worker through pann_range_search. Each request's answer equals the same
 * request run alone (pann_search / pann_range_search). While a server runs it
 * is the only user of its index. */
typedef struct pann_server pann_server;

typedef struct {
  uint32_t max_batch_queries; /* queries per in-flight batch (also the largest k-NN request) */
  uint32_t inflight;          /* batches on the GPU at once, 1..16 */
  uint32_t max_k, max_beam;   /* bounds of k-NN requests */
  uint64_t limit;             /* QueryParams.limit of every k-NN request */
  uint32_t degree_limit;
  double batch_factor;
  int32_t precision;          /* PANN_PREC_*; low precision needs pann_index_set_precision first */
  uint32_t parents;           /* pann_search_options::parents of every k-NN request */
  uint32_t scorer;            /* pann_search_options::scorer of every k-NN request */
  uint64_t scratch_bytes;     /* device scratch of each slot; 0: what max_batch_queries queries at max_k and
                                 max_beam need. A request that alone needs more is refused at submission. */
} pann_server_options;

int pann_server_create(pann_server** out, pann_index* idx, const pann_server_options* opt, const uint32_t* starts,
                       uint32_t n_start);
/* Queries are copied at submission (host memory, nq rows). *ticket names the request. */
int pann_server_submit_knn(pann_server* s, const void* queries, uint32_t nq, uint32_t k, uint32_t beam,
                           uint64_t* ticket);
int pann_server_submit_range(pann_server* s, const void* queries, uint32_t nq, const pann_range_params* rp,
                             uint32_t start_point, uint64_t* ticket);
/* Block until the request is answered, copy its results (k-NN: nq x k ids and
 * distances; range: nq + 1 offsets and the ids, as pann_range_search) and
 * release the ticket. Any output may be NULL. latency_s = submission to
 * answer in host memory. */
int pann_server_wait_knn(pann_server* s, uint64_t ticket, uint32_t* out_ids, float* out_dists, double* latency_s);
int pann_server_wait_range(pann_server* s, uint64_t ticket, uint64_t* out_offsets, uint32_t* out_ids, uint64_t ids_cap,
                           double* latency_s);
/* Requests and queries answered, seconds elapsed, median and 99th-percentile
 * latency since the last reset (reset != 0 starts a new window). */
int pann_server_stats(pann_server* s, int reset, uint64_t* requests, uint64_t* queries, double* seconds, double* p50_s,
                      double* p99_s);
/* Open-loop load generator: request i (k-NN if kind[i] == 0, else range with
 * *rp from range_start) is submitted arrival_s[i] seconds after the call
 * starts, with nq[i] queries from row q_row[i] of query_pool; waits for all.
 * out_latency_s[i] gets each latency, *out_wall_s the time to the last answer. */
int pann_server_replay(pann_server* s, uint32_t nreq, const double* arrival_s, const uint32_t* kind,
                       const uint32_t* nq, const uint32_t* k, const uint32_t* beam, const uint64_t* q_row,
                       const void* query_pool, const pann_range_params* rp, uint32_t range_start, double* out_latency_s,
                       double* out_wall_s);
/* Admission since the last reset: batches launched, queries they held, the
 * largest scratch a batch used and each slot's scratch bytes. */
int pann_server_admission(pann_server* s, int reset, uint64_t* batches, uint64_t* queries, uint64_t* scratch_peak,
                          uint64_t* scratch_bytes);
int pann_server_destroy(pann_server* s);

/* ---------------------------------------------------------------- build */

/* Vamana batch-insertion build into the index's graph (knn_index::build_index,
 * index.h:150-186, batch_insert :188-319). perm (host, length n) is the
 * insertion order; NULL derives it from bp->perm_seed (points ordered by
 * splitmix64(seed + i)). stats may be NULL. */
int pann_build(pann_index* idx, const pann_build_params* bp, const uint32_t* perm, pann_build_stats* stats);

/* ---------------------------------------------------------------- brute force */

/* Exact top-k by full scan (data_tools/compute_groundtruth.cpp:22-60):
 * integer types in exact integer arithmetic, float in FP64. Ties ordered by id.
 * Host buffers; out_dists may be NULL. */
int pann_groundtruth(pann_index* idx, const void* queries, uint32_t nq, uint32_t k, uint32_t* out_ids,
                     double* out_dists);

/* Exact range groundtruth by full scan (compute_range_groundtruth,
 * data_tools/compute_range_groundtruth.cpp:14-30): answer i = every base id j,
 * in increasing order, whose distance to query i as Point::distance computes
 * it (a float) is <= radius (a float, as the tool's -r). Host buffers: answer
 * i is out_ids[out_offsets[i] .. out_offsets[i+1]) (out_offsets has nq + 1
 * entries). With too little room (out_ids NULL and ids_cap 0 to learn the
 * size), out_offsets is filled, PANN_EOVERFLOW returned, and the answers stay
 * on the device for pann_range_fetch, as after pann_range_search. At most
 * 524280 queries per call. */
int pann_range_groundtruth(pann_index* idx, const void* queries, uint32_t nq, float radius, uint64_t* out_offsets,
                           uint32_t* out_ids, uint64_t ids_cap);

/* ---------------------------------------------------------------- misc */

/* Message of the last failing call on this thread ("" if none). */
const char* pann_last_error(void);

/* Seeded synthetic mixture data (host, deterministic, multi-threaded):
 * n x d rows from `components` Gaussian centres. dtype PANN_U8: centres
 * uniform in [lo, hi] per dimension, values rounded and clipped to [0,255];
 * PANN_F32: centres N(0,1) per dimension, rows L2-normalised when normalize.
 * stream 0 = base points, 1 = queries (independent draws, same centres). */
int pann_synth_mixture(int dtype, uint64_t n, uint32_t d, uint32_t components, uint64_t seed,
                       uint32_t stream, double lo, double hi, double sigma, int normalize, void* out);

#ifdef __cplusplus
}
#endif
#endif /* PARLAYANN_B200_H_ */
