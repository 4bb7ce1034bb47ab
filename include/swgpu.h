/*
 * swgpu — B200 engine for MNHN-Tree-Tools' all-pairs Smith-Waterman
 * neighbourhood path.  Plain C ABI: plain pointers and sizes, no C++ or torch
 * types.
 *
 * The reference has no engine API: its OpenCL queue, kernel launches and
 * thresholding sit inline in dbscan.c (opencl_initialization :97-284,
 * region_query :471-522, MPI split :309-468).  These calls replace that inline
 * code; the reference-named functions in mnhn_dropin.h are built on them.
 *
 * Every call returns an swe_status (0 = SWE_OK).  Nothing here exits the
 * process.  A context owns one CUDA stream on one device; use one context per
 * host thread (calls on one context are not thread-safe).
 */
#ifndef SWGPU_H
#define SWGPU_H

#include <stddef.h>
#include <stdint.h>
#include <stdio.h>
#include "mnhn_types.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  SWE_OK = 0,
  SWE_ERR_INVALID = 1,    /* bad argument or input */
  SWE_ERR_CUDA = 2,       /* CUDA runtime error */
  SWE_ERR_OOM = 3,        /* device or host allocation failed */
  SWE_ERR_NO_DEVICE = 4,  /* no usable CUDA device */
  SWE_ERR_TIMEOUT = 5,    /* a bounded device-side wait gave up */
  SWE_ERR_RERUN = 6,      /* the 32-bit rerun queue overflowed */
  SWE_ERR_STATE = 7,      /* call out of order (e.g. no dataset uploaded) */
  SWE_ERR_IO = 8,         /* file could not be read or written */
  SWE_ERR_SWEEP = 9       /* adaptive sweep cannot reach one cluster */
} swe_status;

typedef struct swe_ctx swe_ctx;

typedef struct {
  int device;          /* CUDA device ordinal */
  int sat_limit;       /* 16-bit maxima >= sat_limit are rescored in 32-bit
                          (0 = default 32000; only tests lower it) */
  int packs_per_block; /* row-sequence pairs per tile (0 = default 32) */
  int threads;         /* threads per CTA of the 16x2 kernel (0 = 256) */
  int inject_timeout;  /* test hook: 1 = the score pass's first tile waits on a
                          copy that is never issued, so its bounded wait runs
                          out and the pass returns SWE_ERR_TIMEOUT */
  int threshold_path;  /* test hook for the eps threshold pass: 0 = automatic
                          (transposed two-pass: H-bit words of H sorted rows,
                          then a gather of those words into original order;
                          path 4 for sets too large for it), 1 = rows read
                          from global memory, 2 = bulk-copied rows with the
                          positions staged in shared memory too, 3 = one
                          bulk-copy row buffer, 4 = bulk-copied rows,
                          double-buffered, 5 / 6 = the transposed pass with
                          blocks of at most 16 / 8 rows */
  int kmer_batch_kb;   /* test hook: device batch of the k-mer calls in KB
                          (0 = 1 GB of counts and 256 MB of text) */
  int max_w;           /* lane split of the 16x2 kernel: each column sequence
                          gets the fewest of 8, 16 or 32 lanes that hold at
                          most max_w columns each (0 = 24, the largest) */
  int dbscan_replay;   /* where swe_adaptive_sets replays each (set, eps)
                          DBSCAN: 0 = automatic (on the device, every
                          instance of a round in one launch), 1 = host threads
                          over bitmaps copied back, 2 = device */
} swe_opts;

typedef struct {
  int64_t n_sequences;
  int64_t n_fast;          /* sequences on the packed 16-bit path */
  int64_t n_exceptional;   /* sequences on the 32-bit path (rare symbols, long, empty) */
  int64_t unique_pairs;    /* n*(n-1)/2 */
  double cells;            /* sum over unique pairs of len_a*len_b */
  double tile_cells;       /* cells the 16x2 kernel actually processed, padding included */
  int64_t reruns;          /* pairs rescored in 32-bit after the saturation guard */
  int64_t n_tiles;
  double ms_score_pass;    /* device time of the last score pass */
  double ms_fast_kernel;   /* device time of the 16x2 kernel inside it */
  double ms_last_neighbors;/* device time of the last eps threshold kernels */
  int64_t last_neighbor_launches; /* threshold kernels timed in ms_last_neighbors */
  int dist_bytes;          /* 2 (uint16 matrix) or 4 */
  int64_t h2d_bytes;       /* host->device bytes since the last upload began */
  int64_t d2h_bytes;       /* device->host bytes since the last upload began */
  int64_t kernel_launches; /* this library's kernel launches since the last upload began */
  double ms_last_batch;    /* host time of the last batched DBSCAN (threshold launch, bitmap copies,
                              order-faithful replays) */
  double ms_last_replay;   /* the longest single replay of that batch */
} swe_stats;

const char* swe_strerror(swe_status s);

swe_status swe_create(swe_ctx** out, const swe_opts* opts /* may be NULL */);
void swe_destroy(swe_ctx* ctx);
/* Message of the last failure on this context (never NULL). */
const char* swe_last_error(const swe_ctx* ctx);

/* Copies n sequences to the device.  seqs[i] must be readable at
   [0 .. lens[i]]; position 0 never takes part in a score and position lens[i]
   does (it is the NUL terminator for C strings), as in smith-waterman.c:56-58. */
swe_status swe_upload(swe_ctx* ctx, const char* const* seqs, const size_t* lens, int n);

/* Copies n sequences forming n_sets independent sets: set k holds the
   sequences [set_first[k], set_first[k+1]) (set_first has n_sets+1 entries,
   set_first[0] = 0, set_first[n_sets] = n, non-decreasing).  One score pass
   then scores every pair inside each set and no pair across sets: the many
   split sets of one cluster-tree level in one launch.  swe_upload is this call
   with one set.  The single-set calls below (swe_copy_distances, swe_neighbors,
   swe_dbscan, swe_adaptive) refuse an upload of several sets with
   SWE_ERR_STATE; their _set forms take the set index, and inside a set
   sequence indices are relative to set_first[set]. */
swe_status swe_upload_sets(swe_ctx* ctx, const char* const* seqs, const size_t* lens, int n,
                           const int* set_first, int n_sets);
int swe_set_count(const swe_ctx* ctx);

/* Point datasets (dbscan_L1 / dbscan_L2, dbscan.c:563-779): n points of
   `dims` float coordinates with values[d][i] = coordinate d of point i (the
   reference dataset's values[dimension][point] layout).  The upload computes
   every pair's distance on the GPU with the reference's float arithmetic
   (L1: sum over d in order of |a_d - b_d|; L2: squared distance accumulated
   over d in order with fused multiply-adds, the reference's AVX/FMA build),
   so the single-set calls below (swe_copy_distances, swe_neighbors,
   swe_dbscan, swe_adaptive and their _set forms with set 0) work on points
   with the reference's neighbour test: d <= eps (L1) or d <= eps*eps (L2).
   swe_copy_distances then returns each distance's float bit pattern;
   swe_score_all_pairs does nothing; calls that score sequences return
   SWE_ERR_STATE until the next sequence upload. */
#define SWE_METRIC_L1 1
#define SWE_METRIC_L2 2
swe_status swe_upload_points(swe_ctx* ctx, const float* const* values, int dims, int n, int metric);

/* One data set's score pass split over processes (one per GPU).  The tiles of
   the pass, in descending cost, go one by one to the least loaded of `nparts`
   groups (swe_lpt_partition), identically in every process, and this context
   scores group `part` plus every pair of the 32-bit path; its other pairs hold
   0xFF bytes.  Each pair is scored by exactly one group, so the bytewise
   minimum of all processes' distance storage (an all-reduce with the minimum
   over bytes, e.g. NCCL's ncclMin on ncclUint8, through swe_distance_copy) is
   the full matrix; after copying it back every call below works as after a
   whole pass.  nparts = 1 (the default) is the whole pass.  Applies to the
   current and later uploads. */
swe_status swe_set_partition(swe_ctx* ctx, int part, int nparts);
/* Bytes of the distance storage of the current upload, and a device-to-device
   copy of it to (to_engine = 0) or from (to_engine = 1) a buffer of that size
   on the context's device. */
int64_t swe_distance_bytes(const swe_ctx* ctx);
swe_status swe_distance_copy(swe_ctx* ctx, void* dev_buf, int to_engine);
/* The assignment swe_set_partition uses: owner[t] for costs cost[0..n) given
   in descending order. */
void swe_lpt_partition(const double* cost, int64_t n, int nparts, int* owner);
/* The order in which the score pass takes its tiles (host only): order[0..n)
   receives the indices of cost[] by descending cost, equal costs in index
   order. */
void swe_cost_order(const double* cost, int64_t n, int* order);
/* The grouping of the prefiltered pass (host only; no counterpart in the
   reference): single linkage over `count` pairs (pairs[2c], pairs[2c+1],
   indices below n) taken in the given order, a join skipped when the two
   groups together would exceed `cap` members; label[i] receives the smallest
   index of i's group. */
void swe_capped_linkage(int n, const int* pairs, int64_t count, int cap, int* label);
/* The exchange of a split pass sized to the result (the counterpart of the
   reference's gather of distance stripes to its master, dbscan.c:374-379,
   457-458): a group's payload is the distance rectangles of its own tiles,
   tile after tile in cost order, each row-major, one stored distance
   (swe_distance_bytes / matrix entries: 2 or 4 bytes) per pair; every
   process can compute every group's payload size from the shared layout.
   swe_partition_bytes   bytes of group `part`'s payload (-1: no such group)
   swe_partition_pack    this context's own payload into dev_buf (after its
                         partitioned score pass)
   swe_partition_unpack  bytes [offset, offset + bytes) of group `part`'s
                         payload, received from its process, written into
                         both triangles of this context's matrix
   After every other group's payload is unpacked the matrix equals a whole
   pass (the pairs of the 32-bit path are scored by every group).  Both calls
   wait for the context's stream.  bench.py --split and swgpu/split_pass.py
   exchange payloads in chunks with all-gathers, sizes checked first. */
int64_t swe_partition_bytes(const swe_ctx* ctx, int part);
swe_status swe_partition_pack(swe_ctx* ctx, void* dev_buf);
swe_status swe_partition_unpack(swe_ctx* ctx, int part, const void* dev_buf, int64_t offset, int64_t bytes);

/* Scores every pair of the uploaded sequences into the device distance matrix
   (one pass; later neighbour/DBSCAN calls reuse it). */
swe_status swe_score_all_pairs(swe_ctx* ctx);

/* n_s x n_s distance matrix of one set (n_s = its size), row-major in the
   set's index order. */
swe_status swe_copy_set_distances(swe_ctx* ctx, int set, uint32_t* out);
/* Rows [row0, row1) of that matrix ((row1-row0) x n_s entries). */
swe_status swe_copy_set_rows(swe_ctx* ctx, int set, int row0, int row1, uint32_t* out);

/* Statistics of the block rows [r0, r1) x columns [c0, c1) of one set's
   distance matrix (indices inside the set), without copying it: per row the
   sum of the distances (row_sum) and the sum of floor((d - mean)^2) with each
   square rounded once in double (row_sqdev), both r1-r0 entries or NULL, and
   the block's smallest and largest distance.  The reductions of
   comparison.c:84-403 (mean, sigma, silhouette, extremes) are built on it. */
swe_status swe_block_stats(swe_ctx* ctx, int set, int r0, int r1, int c0, int c1, double mean, uint64_t* row_sum,
                           uint64_t* row_sqdev, uint32_t* min, uint32_t* max);

/* Copies the n x n distance matrix to host memory (out holds n*n entries). */
swe_status swe_copy_distances(swe_ctx* ctx, uint32_t* out);

/* eps-neighbourhoods of every point, the reference's region_query
   (dbscan.c:525-561) for all points at once: ascending indices k with
   (float)d(k,i) <= eps, i itself included.  *row_ptr (n+1 entries) and *cols
   are malloc'd; release them with swe_free. */
swe_status swe_neighbors(swe_ctx* ctx, float eps, int64_t** row_ptr, int** cols);

/* DBSCAN at one eps (dbscan.c:950-1047 semantics) on the scored matrix.
   The split set is malloc'd reference-style. */
swe_status swe_dbscan(swe_ctx* ctx, float eps, int minpts, split_set* out);

/* Adaptive sweep (dbscan.c:1117-1380 semantics) on the scored matrix.  Log
   lines go to `log` (stdout when NULL); split sets are written to
   <prefix>%04d unless prefix is NULL.  If out_sets is not NULL it receives a
   malloc'd array of the kept layers (free each with
   free_split_set_and_associated_clusters, then the array with swe_free);
   out_n_sets (if not NULL) receives their number. */
swe_status swe_adaptive(swe_ctx* ctx, float eps_start, float eps_inc, int minpts, const char* prefix,
                        FILE* log, split_set** out_sets, int* out_n_sets);

/* The same three calls on one set of a several-set upload. */
swe_status swe_neighbors_set(swe_ctx* ctx, int set, float eps, int64_t** row_ptr, int** cols);
swe_status swe_dbscan_set(swe_ctx* ctx, int set, float eps, int minpts, split_set* out);
swe_status swe_adaptive_set(swe_ctx* ctx, int set, float eps_start, float eps_inc, int minpts, const char* prefix,
                            FILE* log, split_set** out_sets, int* out_n_sets);

/* Result of one set's sweep in swe_adaptive_sets. */
typedef struct {
  int status;          /* swe_status of this set's sweep */
  int truncated;       /* 1 when max_steps ended the sweep before a one-cluster result */
  int steps;           /* DBSCAN runs of the sweep phase (after the starting eps) */
  int n_layers;        /* kept layers */
  split_set* layers;   /* malloc'd array of the kept layers */
  char* log;           /* malloc'd NUL-terminated log text of the sweep (the lines
                          swe_adaptive would print for this set alone) */
  double done_ms;      /* host milliseconds from the call's start to this set's end */
} swe_sweep_result;

/* Adaptive sweeps of every uploaded set at once (the cluster tree's split
   sets of one level).  Each set runs the sweep of swe_adaptive_set with the
   same parameters, bounded to max_steps DBSCAN runs after the starting eps
   (0 = unbounded, as in the reference).  The sweeps advance in rounds: each
   round one threshold launch serves the pending eps values of every active
   set, then host threads replay the DBSCAN runs and advance the sweeps.  A
   set's layers and log equal what swe_adaptive_set would produce for it with
   the same bound.  With prefix not NULL, set k's layers are stored as
   <prefix><k>_%04d.  results holds swe_set_count() entries; release them
   with swe_free_sweep_results.  The call fails only on CUDA or allocation
   errors; a set whose sweep fails has its own status. */
swe_status swe_adaptive_sets(swe_ctx* ctx, float eps_start, float eps_inc, int minpts, int max_steps,
                             const char* prefix, swe_sweep_result* results);
void swe_free_sweep_results(swe_sweep_result* results, int n);

/* Distances of one query to every uploaded sequence (out holds n entries).
   q must be readable at [0 .. qlen]. */
swe_status swe_score_one_to_many(swe_ctx* ctx, const char* q, size_t qlen, unsigned* out);

/* Distances of explicit pairs of uploaded sequences. */
swe_status swe_score_pairs(swe_ctx* ctx, const int* a, const int* b, int64_t npairs, unsigned* out);

swe_status swe_get_stats(const swe_ctx* ctx, swe_stats* out);

/* DBSCAN replay (dbscan.c:950-1047 order semantics) on caller-provided
   neighbourhoods; host only, no GPU involved.  Row i of `bits` is
   words_per_row 64-bit words with bit k set iff k is an eps-neighbour of i
   (i itself included when eps >= 0); counts[i] is that row's popcount. */
swe_status swe_dbscan_bitmap(int n, const uint64_t* bits, int words_per_row, const int* counts, int minpts,
                             split_set* out);

/* The same replay for many independent instances in one device launch (one
   warp each, the traversal swe_adaptive_sets uses on the device): instance k
   has n[k] points, rows of (n[k] + 63) / 64 words starting at word
   bits_off[k] of `bits`, counts starting at counts_off[k] of `counts` (host
   arrays, copied to the device).  out[k] as swe_dbscan_bitmap's. */
swe_status swe_dbscan_bitmaps_device(swe_ctx* ctx, int n_inst, const int* n, const uint64_t* bits,
                                     const int64_t* bits_off, int64_t bits_words, const int* counts,
                                     const int64_t* counts_off, int64_t counts_len, int minpts, split_set* out);

/* The adaptive sweep (dbscan.c:1117-1380 semantics) over a distance matrix the
   caller holds (row-major n x n, the neighbour test (float)d <= eps); host
   only, no GPU involved.  batch is the number of eps values evaluated per
   round; with speculate != 0 the round of the starting eps also evaluates the
   sweep batch that follows it (the engine's sweeps do both).  Log, files and
   out_sets as swe_adaptive. */
swe_status swe_adaptive_matrix(int n, const uint32_t* D, float eps_start, float eps_inc, int minpts,
                               const char* prefix, FILE* log, int speculate, int batch, split_set** out_sets,
                               int* out_n_sets);

/* Measures, on `device`, the issue rate of the 16x2 kernel's per-cell
   instruction mix (one PRMT, three packed add-max, one packed max) on
   independent chains: *cells_per_s DP cells per second (two per packed
   update) and *lane_instr_per_s the corresponding 32-bit-lane instructions
   per second.  The integer roofline of the score pass is derived from it. */
swe_status swe_measure_mix_peak(int device, double* cells_per_s, double* lane_instr_per_s);

/* Step timer on the context's stream: start records a CUDA event, stop
   records a second one, waits for it and returns the elapsed milliseconds.
   Host work between the two calls (DBSCAN replay) is inside the interval. */
swe_status swe_timer_start(swe_ctx* ctx);
swe_status swe_timer_stop(swe_ctx* ctx, double* ms);

/* Tile-plan autotuner.  No counterpart in the reference, whose OpenCL launch
   leaves the work-group size to the driver (dbscan.c:497-501, local size
   NULL) and whose kernel has no tiles.

   The 16x2 kernel's plan is three knobs: row packs (two sequences each) per
   tile, threads per CTA, and the lane split (a column sequence gets the
   fewest of 8, 16 or 32 lanes that hold at most max_w columns each).  Every
   plan computes the same distances; their speed depends on the device and on
   the length distribution.  swe_autotune takes a length-stratified sample of
   up to 4,096 of the given sequences, scores it on a scratch context of the
   same device with each candidate plan (packs 16 / 32 / 64, threads 128 /
   256, max_w 16 / 20 / 24), checks that every plan's matrix equals the
   default plan's, and keeps the fastest unless it is within 2 % of the
   default, which is then kept.  The plan is
   set on ctx: it applies to the next upload, and an upload ctx already holds
   is laid out again (its distances must be scored again).

   cache_path   NULL, or a text file of "key packs threads max_w" lines: a
                line with this key is used without timing anything
                (SWE_TUNE_FORCE times anyway); a newly timed plan is appended
   key          device name, SM count, the sample size class and the length
                histogram (sixteen 64-symbol bins, in twentieths) */
#define SWE_TUNE_FORCE 1
typedef struct {
  int packs_per_block, threads, max_w;  /* the chosen plan */
  int from_cache;                       /* 1: read from cache_path, nothing timed */
  int candidates;                       /* plans timed */
  int sample;                           /* sequences in the timing sample */
  double sample_cells;                  /* DP cells of one pass over the sample */
  double ms_default;                    /* 16x2 kernel time of the default plan (32, 256, 24) */
  double ms_best;                       /* 16x2 kernel time of the chosen plan */
  char key[160];
} swe_tune_result;
swe_status swe_autotune(swe_ctx* ctx, const char* const* seqs, const size_t* lens, int n, const char* cache_path,
                        int flags, swe_tune_result* out);

/* Allocation-free scoring of explicit pairs.  No counterpart in the reference
   (which has no device API at all).

   For callers that cannot allocate device memory: real-time or embedded hosts
   that must not call the device allocator once they have started, and programs
   whose device memory is all owned by their own pooling allocator, which this
   library can neither see nor grow.  The caller passes device buffers it
   already owns; this call calls no cudaMalloc, cudaFree or other allocating
   routine.

   seqs         device bytes; sequence i is the C string at seqs + off[i] of
                length len[i] (readable at [0 .. len[i]], scored like score())
   off, len     device arrays indexed by sequence
   pairs        device int array of 2*npairs indices (a, b)
   out          device array of npairs distances
   max_len      upper bound on every len[i] the pairs reference,
                at most SWE_NOALLOC_MAX_LEN (larger values: SWE_ERR_INVALID)
   stream       cudaStream_t to run on (NULL: the default stream)

   The call waits for `stream` and returns when `out` holds the distances.  A
   pair that references a sequence longer than max_len is not scored: its
   distance reads 0xFFFFFFFF and the call returns SWE_ERR_INVALID (every other
   pair is still scored).  An error that earlier work of the caller left
   pending in the CUDA runtime is returned as SWE_ERR_CUDA before anything
   runs, and stays pending for the caller.

   Long sequences need scratch, which is one fixed 4 MiB device array per GPU
   (kept until the process exits), so a call runs at most 2^20/(max_len+1)
   warps.  Every call on a device shares that array and it keeps the last
   call's contents (each call writes every word before reading it, and clears
   its counter of over-length pairs): calls that overlap on the GPU - on
   different streams or threads - race and must be serialised by the caller.
   The first call on a device looks up the array's device address with that
   device current and keeps it with the CUDA context current then (a call from
   another context of the device looks it up again); make that first call
   before any stream capture, and do not call it again after a
   cudaDeviceReset of the device. */
#define SWE_NOALLOC_MAX_LEN 65535
swe_status swe_score_pairs_noalloc(const char* seqs, const int64_t* off, const int* len, const int* pairs,
                                   int64_t npairs, unsigned* out, int max_len, void* stream);

/* ------------------------------------------------------------------------
   Learned prefilter (no counterpart in the reference).  Features are the
   5-mer counts of kmers.c (windows 0 .. len-6, A0 C1 G2 T3, windows with other
   symbols count nothing), L1-normalised; an MLP 1024 -> 512 -> 256 -> 128 with
   exact GELU after the first two layers, bf16 weights and fp32 accumulation,
   maps them to embeddings whose L2 distance is trained (MSE) to predict
   d / (4 * max(len_a, len_b)) of the exact distance d.  The exact engine
   stays the default; the prefilter only decides which pairs to score.
   ------------------------------------------------------------------------ */

/* k-mer features (k = 1..6) of the uploaded sequences: out holds n * 4^k
   floats (row i = sequence i), or NULL to only compute them. */
swe_status swe_kmer_features(swe_ctx* ctx, int k, float* out);

/* Random initial weights (uniform +-1/sqrt(fan_in), seeded). */
swe_status swe_prefilter_init(swe_ctx* ctx, uint64_t seed);
/* Number of parameters: W1 [512x1024], b1, W2 [256x512], b2, W3 [128x256], b3,
   in that order, row-major, in one flat fp32 vector. */
int64_t swe_prefilter_param_count(void);
/* Copies the fp32 master parameters out (get != NULL) and/or in (set != NULL). */
swe_status swe_prefilter_params(swe_ctx* ctx, float* get, const float* set);
/* Mean loss over the pairs (a[k], b[k]) with exact distances dist[k], and
   the gradient of every parameter (same layout as the parameters). */
swe_status swe_prefilter_loss_grad(swe_ctx* ctx, const int* a, const int* b, const unsigned* dist, int npairs,
                                   float* loss, float* grad);
/* Adam training (decoupled weight decay weight_decay, 0 for none) over the
   pairs for `epochs` passes in shuffled batches of batch_pairs pairs (full
   batches only); epoch_loss[e] = mean batch loss.  The squared error of a
   pair whose distance is within over_eps (an eps-neighbour) counts
   over_weight times when the embedding distance over-estimates it (1 = plain
   mean squared error): the candidate test's margins are set by such
   over-estimates. */
swe_status swe_prefilter_train(swe_ctx* ctx, const int* a, const int* b, const unsigned* dist, int64_t npairs,
                               int epochs, int batch_pairs, float lr, float weight_decay, uint64_t seed,
                               float over_eps, float over_weight, float* epoch_loss);
/* Embeddings of the uploaded sequences (out: n x 128, or NULL). */
swe_status swe_prefilter_embed(swe_ctx* ctx, float* out);
/* Embedding distances of explicit pairs. */
swe_status swe_prefilter_pair_dist(swe_ctx* ctx, const int* a, const int* b, int64_t np, float* out);
/* Replaces the embeddings of the uploaded sequences (n x 128) by the
   caller's, e.g. an embedding without the network for comparison; the next
   swe_prefilter_embed recomputes them from the network. */
swe_status swe_prefilter_set_embeddings(swe_ctx* ctx, const float* emb);

typedef struct {
  int64_t candidates;   /* pairs passing the length bound and the embedding margin */
  int64_t tiles_kept;   /* tiles of the 16x2 kernel that hold a candidate */
  int64_t tiles_all;    /* tiles of the full layout */
  double tile_cells;    /* DP cells the 16x2 kernel processed */
  double ms_embed, ms_candidates, ms_layout, ms_score, ms_total;  /* host wall times */
  int fallback_full;    /* 1 when there were too many candidates and every pair was scored */
  double ms_groups;     /* of ms_layout: candidate groups and the sort keys */
  double ms_marks;      /* of ms_layout: marking the tiles that hold a candidate */
  double ms_upload;     /* of ms_layout: layout arrays to the device and the selector build */
} swe_prefilter_stats;

/* Margins of the prefilter by the pair's longer length L: bucket b < n-1
   holds L < upper[b], the last bucket every longer pair (upper[n-1] unused). */
#define SWE_MARGIN_BUCKETS 8
typedef struct {
  int n;
  int upper[SWE_MARGIN_BUCKETS];
  float margin[SWE_MARGIN_BUCKETS];
} swe_margins;

/* Prefiltered score pass for neighbourhoods up to eps: a pair is scored
   exactly when 4*|len_a - len_b| <= floor(eps) (every distance is at least
   that) and, with use_emb, its embedding distance is at most
   floor(eps) / (4*max(len_a, len_b)) + margin(max(len_a, len_b)).
   Sequences joined by candidate pairs that pass without margin are grouped
   (connected components), each group laid out contiguously, and only the
   tiles of the 16x2 kernel that hold a candidate pair are run; every other pair reads as the largest
   distance (never an eps-neighbour).  Scores that are computed are exact, so
   neighbourhoods at any eps' <= eps are a subset of the exact ones, missing
   only pairs the prefilter skipped.  swe_score_all_pairs returns to the exact
   pass. */
swe_status swe_score_prefiltered(swe_ctx* ctx, float eps, const swe_margins* margins, int use_emb,
                                 swe_prefilter_stats* out);

/* The tensor-core GEMM alone, for tests: C[M x N] = A[M x K] * B[N x K]^T
   (+ bias, GELU when act = 1) with A, B bf16 and C fp32 DEVICE pointers;
   M and N multiples of 128, K a multiple of 64. */
swe_status swe_gemm_bf16(int device, const void* A, const void* B, int M, int N, int K, const float* bias, int act,
                         float* C);

/* ------------------------------------------------------------------------
   k-mer frequency tables of fasta2kmer (kmers.c:157-389).  Independent of
   the uploaded dataset: sequences are passed in and counted on the GPU.
   ------------------------------------------------------------------------ */

#define SWE_KMER_MAX_DNA 15     /* gen_dna_kmers builds its table with int shifts (kmers.c:87-107) */
#define SWE_KMER_MAX_PROTEIN 7  /* 20^7 counts per sequence; longer k-mers exceed any row the reference allocates */

/* Number of k-mers: 4^k (kmers.c:65-73) or 20^k with protein != 0
   (kmers.c:75-83); 0 when k is outside 1..SWE_KMER_MAX_DNA / _PROTEIN. */
int64_t swe_kmer_count(int k, int protein);

/* Counts of every k-mer in the sequences seqs[i], len[i] bytes each (the
   caller passes strlen, kmers.c:162).  Semantics of
   frequence_of_kmer_in_sequence (kmers.c:157-241) for each table entry:
   windows start at 0 .. len-k-1 (the window ending at the last symbol is never
   counted, and len <= k gives all zeros), symbols compare as raw bytes
   against 'A','C','G','T' (index bits 2p..2p+1 = symbol p, A0 C1 G2 T3,
   kmers.c:26-107) or, with protein != 0, against the 20 letters
   ACDEFGHIKLMNPQRSTVWY (index = base-20 number with symbol 0 most
   significant, kmers.c:109-155), and a count keeps the low 16 bits of the
   true count as a signed short.  Row i of the result goes to rows[i]
   (swe_kmer_count(k, protein) shorts). */
swe_status swe_kmer_counts(swe_ctx* ctx, const char* const* seqs, const int64_t* len, int64_t n, int k, int protein,
                           int16_t* const* rows);

/* Receives consecutive pieces of a text; returns 0 to go on, else stops the
   producer (which then returns SWE_ERR_IO). */
typedef int (*swe_text_sink)(const char* data, size_t size, void* user);

/* The text write_kmer_base prints for a frequency table (kmers.c:373-385):
   per row i "sequence_<i>" then each count as "%hi", separated by tabs,
   ending in a newline.  The digits are formatted on the GPU; the text is
   handed to `sink` in pieces in order. */
swe_status swe_kmer_tsv(swe_ctx* ctx, const int16_t* const* rows, int64_t n, int64_t nk, swe_text_sink sink,
                        void* user);

/* ---- kmer2pca: principal components of a sample x feature table ----------
   `data` is n_samples rows of n_features doubles, row-major (kmer2pca.c's
   in_data, filled by data_from_file, kmer2pca.c:255-268).  The covariance is
   the reference's (kmer2pca.c:337-481): means over all samples, sums over the
   first n_samples - n_samples % 4 samples (its AVX loop never adds the last
   n_samples % 4), divided by n_samples.  Tables of integers in the int16
   range (every fasta2kmer table) are kept as int16 on the GPU and their
   covariance is the exact value rounded (see csrc/pca.cu); other tables are
   centred and summed in float64. */
typedef struct {
  int exact;            /* 1: integer table, covariance from exact integer sums */
  int64_t h2d_bytes;    /* table bytes copied to the GPU */
  double ms_upload;     /* host time of the table check, conversion and copy */
  double ms_covariance; /* device time of the covariance kernels */
  double ms_gram;       /* device time of the Gram tile kernel inside it */
  double ms_eigen;      /* host time of the eigen-decomposition call (swe_pca) */
  double ms_project;    /* device time of the projection kernel */
} swe_pca_info;

/* means_from_data + feature_covariance_matrix (kmer2pca.c:286-481): cov gets
   the n_features x n_features covariance matrix (row-major, symmetric).  The
   table stays on the GPU for a following swe_pca_project with data == NULL.
   info may be NULL. */
swe_status swe_pca_covariance(swe_ctx* ctx, const double* data, int64_t n_samples, int64_t n_features, double* cov,
                              swe_pca_info* info);

/* eigen_from_corr (kmer2pca.c:107-138, LAPACK dsyev): every eigenvalue of the
   symmetric cov in ascending order into eigenvalues[n_features], and the unit
   eigenvectors of the n_vectors largest ones, largest first, into
   vectors[n_vectors][n_features] (n_vectors may be 0, vectors then unused).
   An eigenvector's sign is not defined by the problem; each is returned with
   its largest-magnitude entry positive.  Host code, no context. */
swe_status swe_pca_eigen(const double* cov, int64_t n_features, int64_t n_vectors, double* eigenvalues,
                         double* vectors);

/* swe_pca_eigen with the O(n_features^3) part on the GPU: the Householder
   reduction (three launches per column, the matrix in device memory) and the
   bisection of every eigenvalue; inverse iteration for the n_vectors wanted
   vectors and their back-transformation on the host.  Same outputs and sign
   rule as swe_pca_eigen, equal to it up to rounding; matrices below 64 x 64
   and diagonal ones are solved on the host. */
swe_status swe_pca_eigen_gpu(swe_ctx* ctx, const double* cov, int64_t n_features, int64_t n_vectors,
                             double* eigenvalues, double* vectors);

/* obtain_projections (kmer2pca.c:141-211): projections[j][i] = sum over k of
   data[j][k] * vectors[i][k] in the order of k (one fused multiply-add per
   term) for the `dimensions` vectors given (1 <= dimensions <= n_features).
   data == NULL projects the table left on the GPU by the previous
   swe_pca_covariance / swe_pca call of this context (same shape). */
swe_status swe_pca_project(swe_ctx* ctx, const double* data, int64_t n_samples, int64_t n_features,
                           const double* vectors, int64_t dimensions, double* projections, swe_pca_info* info);

/* The whole of kmer2pca after reading its file (kmer2pca.c:540-586): one
   table upload, the covariance, the eigen-decomposition (swe_pca_eigen_gpu)
   and the projections onto the eigenvectors of the `dimensions` largest
   eigenvalues.
   eigenvalues[n_features] ascending, projections[n_samples][dimensions]. */
swe_status swe_pca(swe_ctx* ctx, const double* data, int64_t n_samples, int64_t n_features, int64_t dimensions,
                   double* eigenvalues, double* projections, swe_pca_info* info);

void swe_free(void* p);

#ifdef __cplusplus
}
#endif
#endif /* SWGPU_H */
