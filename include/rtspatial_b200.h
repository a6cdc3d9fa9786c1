/*
 * rtspatial_b200 — C ABI of the B200-native spatial index.
 *
 * Drop-in boundary for rtspatial::SpatialIndex<float, 2>
 * (include/rtspatial/spatial_index.cuh:62-931 in the RTSpatial project): the
 * same operations (Init/Clear/Insert/Delete/Update/Query), the same input
 * layouts (Envelope<Point<float,2>> = 4 floats min.x, min.y, max.x, max.y;
 * Point<float,2> = 2 floats), the same implicit insertion-order ids and the
 * same result contract: one (geom_id, query_id) pair per match, handed to a
 * counting or collecting handler.  Plain pointers and sizes only.
 *
 * Conventions
 *  - Array arguments are device pointers, or pinned host pointers the device
 *    can address (the reference's tests pass pinned host vectors,
 *    test/test_point_queries.h:67-84).
 *  - `stream` is a cudaStream_t (NULL = legacy default stream).  Calls are
 *    asynchronous with respect to the host unless noted.
 *  - Every call returns RTS_OK or an error code; rts_last_error() gives a
 *    per-thread message.  Nothing aborts the process (the reference aborts or
 *    throws, spatial_index.cuh:387-389).
 *  - Coordinates must be finite.  The contains predicates are exact for any
 *    finite input; range-intersects is exact for finite inputs.
 */
#ifndef RTSPATIAL_B200_H
#define RTSPATIAL_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define RTS_OK 0
#define RTS_ERR_INVALID_ARGUMENT 1
#define RTS_ERR_CUDA 2
#define RTS_ERR_OUT_OF_MEMORY 3
#define RTS_ERR_QUEUE_FULL 4   /* a collecting queue received more pairs than its capacity */
#define RTS_ERR_CAPACITY 5     /* a size exceeds a documented maximum */
#define RTS_ERR_UNSUPPORTED 6
#define RTS_ERR_TIMEOUT 7      /* a wait ended before the request was done */

/* ---- predicates: values of rtspatial::Predicate (geom/predicates.h:7-10) - */
#define RTS_PREDICATE_INTERSECTS 0
#define RTS_PREDICATE_CONTAINS 1

/* ---- handlers ------------------------------------------------------------
 * The reference selects a device handler at shader compile time
 * (CMakeLists.txt:73-104 force-includes default_handlers/*.h).  Here the
 * handler is a run-time argument: the same two shipped behaviours, built in,
 * or the caller's own functions from a handler module (below):
 *  RTS_HANDLER_COUNT   arg = unsigned long long* in device memory; each pair
 *                      adds 1 (default_handlers/counting_handlers.h:7-25).
 *  RTS_HANDLER_COLLECT arg = rts_queue* in device memory; each pair is
 *                      appended (default_handlers/collecting_handlers.h:9-31,
 *                      utils/queue.h:22-27).  Pairs beyond `capacity` are not
 *                      written but still counted in *size, so after the query
 *                      *size > capacity signals overflow and gives the size
 *                      needed. */
#define RTS_HANDLER_COUNT 0
#define RTS_HANDLER_COLLECT 1
/* RTS_HANDLER_MODULE  the caller's own rtspatial_handle_* device functions,
 *                      called once per pair with `arg`, from the handler module
 *                      loaded by rts_load_handler_module (the reference's
 *                      compile-time handler header, CMakeLists.txt:73-104).
 *                      Batches of one launch either all use it or none does. */
#define RTS_HANDLER_MODULE 2

/* thrust::pair<uint32_t, uint32_t> as the collecting handler writes it. */
typedef struct rts_pair {
  uint32_t geom_id;
  uint32_t query_id;
} rts_pair;

/* Device-side queue with the member layout of
 * rtspatial::dev::Queue<thrust::pair<uint32_t,uint32_t>> (utils/queue.h:60-62:
 * ArrayView<T>{T* data; size_t size;} followed by uint32_t* last_pos). */
typedef struct rts_queue {
  rts_pair* data;
  uint64_t capacity;
  uint32_t* size;
} rts_queue;

/* thrust::pair<size_t, Envelope<Point<float,2>>> as Update takes it
 * (spatial_index.cuh:280-281): 8-byte id, then the envelope. */
typedef struct rts_update_entry {
  uint64_t id;
  float min_x, min_y, max_x, max_y;
} rts_update_entry;

/* thrust::pair<size_t, Envelope<Point<double,2>>> for a double index
 * (SpatialIndex<double, 2>, spatial_index.cuh:280-281). */
typedef struct rts_update_entry_f64 {
  uint64_t id;
  double min_x, min_y, max_x, max_y;
} rts_update_entry_f64;

/* ---- configuration ---------------------------------------------------------
 * First block: the fields of rtspatial::Config (spatial_index.cuh:22-37),
 * accepted for source compatibility.  ptx_root is not a field here: the C++
 * drop-in loads the handler module from it (rts_load_handler_module); the
 * OptiX build flags and the intersects cost-model fields do not change results
 * and are ignored.
 * Second block: this library's own structure and traversal knobs. */
typedef struct rts_config {
  uint64_t max_geometries;      /* capacity reserved when preallocate != 0 */
  uint64_t max_queries;         /* accepted, no effect */
  int32_t preallocate;
  int32_t prefer_fast_build_geom;  /* accepted, no effect */
  int32_t prefer_fast_build_query; /* accepted, no effect */
  int32_t compact;                 /* accepted, no effect */
  float geom_sample_rate;          /* accepted, no effect */
  float query_sample_rate;         /* accepted, no effect */
  float intersect_cost_weight;     /* accepted, no effect */
  uint32_t max_geom_samples;       /* accepted, no effect */
  uint32_t max_query_samples;      /* accepted, no effect */
  uint32_t max_parallelism;        /* accepted, no effect */

  int32_t node_width;     /* children per node and boxes per leaf: 4, 8, 16 or 32 (default 16) */
  int32_t traversal;      /* RTS_TRAVERSAL_* */
  int32_t curve;          /* RTS_CURVE_*: the order leaves are packed in */
  int32_t max_trees;      /* sub-trees kept before a merge (1..16, default 4): the sub-trees
                             beside the largest merge into one when they hold at most an
                             eighth of its slots and fit in the slot arrays, else every box
                             is re-sorted into one tree */
  float rebuild_fraction; /* an insert batch larger than this fraction of the index rebuilds everything */
  int32_t sort_queries;   /* visit queries in curve order (results keep the caller's query ids):
                             0 never, 1 always, 2 when a launch has >= 8192 queries */
  float rebuild_update_fraction; /* updates since the last rebuild, as a fraction of the index,
                                    above which Update re-sorts every box (below it, envelopes
                                    are written in place or moved to a new sub-tree) */
  uint32_t chunk;         /* queries per device work item (0 = library default) */
  int32_t query_occupancy; /* 2 / 3 / 4: query kernel capped at 128 / 80 / 64 registers
                              (2 / 3 / 4 CTAs of 256 threads per SM); 1: uncapped; 0: per
                              scheme (thread 2, packet 4, team 1) */
  float frontier_factor;   /* frontier traversal: entries per query of each level buffer
                              (queries beyond it are answered depth-first); 0 = 16 */
  int32_t coord_bits;      /* 32: SpatialIndex<float, 2>; 64: SpatialIndex<double, 2>, whose
                              envelopes, points and updates go through the _f64 calls */
  int32_t group_loads;     /* RTS_LOADS_*: how the thread scheme's node-group loads use L1 */
} rts_config;

#define RTS_LOADS_AUTO 0      /* streaming for collecting (and user-handler) launches once the
                                 stored envelopes pass 64 MB; cached otherwise */
#define RTS_LOADS_CACHED 1    /* groups are cached in L1 (small, hot trees) */
#define RTS_LOADS_STREAMING 2 /* groups bypass L1 allocation (L1::no_allocate) and fetch whole
                                 256-byte L2 lines: L1 keeps the kernel's own working set */

#define RTS_TRAVERSAL_AUTO 0   /* packet for range-intersects launches, thread otherwise */
#define RTS_TRAVERSAL_THREAD 1 /* one thread per query, loops over a node's children */
#define RTS_TRAVERSAL_TEAM 2   /* node_width lanes per query, one child per lane */
#define RTS_TRAVERSAL_FRONTIER 3 /* level by level over the whole launch (batches of one
                                    predicate and handler; others run depth-first) */
#define RTS_TRAVERSAL_PACKET 4 /* one warp walks a packet of up to 32 queries, one entry
                                  per lane; best with sorted queries */
#define RTS_TRAVERSAL_STAGED 5 /* one thread per query; each visited node group (and a
                                  leaf group's ids) is bulk-copied into shared memory
                                  (node_width <= 16; wider indexes use THREAD) */

#define RTS_CURVE_MORTON 0
#define RTS_CURVE_HILBERT 1

typedef struct rts_index rts_index;

/* Fills `cfg` with the reference's defaults (spatial_index.cuh:22-37) and this
 * library's defaults for the remaining fields. */
int rts_config_default(rts_config* cfg);

/* SpatialIndex::Init (spatial_index.cuh:83-110). */
int rts_create(const rts_config* cfg, rts_index** out);
int rts_destroy(rts_index* index);

/* SpatialIndex::Clear (spatial_index.cuh:118-129): drops every box; ids
 * restart at 0. */
int rts_clear(rts_index* index, void* stream);

/* SpatialIndex::Insert (spatial_index.cuh:142-196): appends n envelopes
 * (n*4 floats); they receive ids size .. size+n-1. */
int rts_insert(rts_index* index, const float* envelopes, uint64_t n, void* stream);

/* SpatialIndex::Delete (spatial_index.cuh:208-265): each listed id becomes
 * Envelope::Invalid() (max := min) and stays indexed; ids >= size are
 * ignored, as the reference's `idx < v_envelopes.size()` guard does. */
int rts_delete(rts_index* index, const uint64_t* ids, uint64_t n, void* stream);

/* SpatialIndex::Update (spatial_index.cuh:280-336): overwrites the listed
 * envelopes.  Every id must be < size (the reference asserts it, :295);
 * out-of-range entries are skipped here; an id listed twice keeps one of its
 * envelopes.  An envelope that stays inside its leaf group's hull is written
 * in place; one that leaves it moves, with its id, to a new sub-tree (the
 * reference refits instead, letting every hull above it grow).  Waits for the
 * stream once (to size that sub-tree). */
int rts_update(rts_index* index, const rts_update_entry* updates, uint64_t n, void* stream);

/* SpatialIndex::Query(Predicate, ArrayView<point_t>, void*, cudaStream_t)
 * (spatial_index.cuh:352-391).  Only RTS_PREDICATE_CONTAINS is defined for
 * points (the reference aborts on any other; this returns
 * RTS_ERR_INVALID_ARGUMENT). */
int rts_query_points(rts_index* index, int predicate, const float* points, uint64_t n,
                     int handler, void* arg, void* stream);

/* ---- double indexes (coord_bits = 64): SpatialIndex<double, 2> -------------
 * The same calls over double envelopes {min.x, min.y, max.x, max.y}, points
 * {x, y} and rts_update_entry_f64 (Insert, Update, Query of
 * spatial_index.cuh:142-515 instantiated for double; rts_delete and the
 * batched / planned / served calls apply unchanged, with the _F64 query
 * kinds).  As in the reference, the contains predicates compare coordinates
 * rounded to float (Point<double,2>::get_coordinate returns float,
 * geom/point.cuh:68-71) while range-intersects runs the ray-slab test in
 * double (details/ray_params.h:169-292).  A float index rejects these calls
 * and a double index rejects the float ones (RTS_ERR_INVALID_ARGUMENT). */
int rts_insert_f64(rts_index* index, const double* envelopes, uint64_t n, void* stream);
int rts_update_f64(rts_index* index, const rts_update_entry_f64* updates, uint64_t n,
                   void* stream);
int rts_query_points_f64(rts_index* index, int predicate, const double* points, uint64_t n,
                         int handler, void* arg, void* stream);
int rts_query_envelopes_f64(rts_index* index, int predicate, const double* envelopes,
                            uint64_t n, int handler, void* arg, void* stream);

/* SpatialIndex::Query(Predicate, ArrayView<envelope_t>, void*, cudaStream_t)
 * (spatial_index.cuh:407-515): RTS_PREDICATE_CONTAINS reports boxes that
 * contain the query box; RTS_PREDICATE_INTERSECTS reports the reference's
 * two-pass ray-slab result set. */
int rts_query_envelopes(rts_index* index, int predicate, const float* envelopes, uint64_t n,
                        int handler, void* arg, void* stream);

/* ---- batched queries ----------------------------------------------------
 * Many Query calls fused into one persistent launch with a device-side work
 * queue.  Each batch keeps its own handler/arg and its own 0-based query ids,
 * so a batch's results equal those of the same Query call made alone.  When
 * the launch sorts its queries, every batch has one predicate and handler,
 * and the handler counts or the traversal is RTS_TRAVERSAL_PACKET, the
 * queries of all batches are sorted together and each result is routed to its
 * batch's handler. */
#define RTS_QUERY_POINTS 0
#define RTS_QUERY_ENVELOPES 1
#define RTS_QUERY_POINTS_F64 2    /* double index: 2 doubles per point */
#define RTS_QUERY_ENVELOPES_F64 3 /* double index: 4 doubles per envelope */
typedef struct rts_batch {
  int32_t query_kind; /* RTS_QUERY_POINTS or RTS_QUERY_ENVELOPES */
  int32_t predicate;  /* RTS_PREDICATE_* */
  const float* queries;
  uint64_t n;
  int32_t handler;
  int32_t reserved;
  void* arg;
} rts_batch;

/* Runs n_batches batches (host array) in one launch.  The descriptors are
 * staged by the library; the call returns once they are enqueued. */
int rts_query_batched(rts_index* index, const rts_batch* batches, uint32_t n_batches,
                      void* stream);

/* ---- prepared launches and CUDA-graph replay -----------------------------
 * No counterpart in the reference (its Query re-packs launch parameters on
 * every call, spatial_index.cuh:359-367).  A plan fixes a set of batches
 * (query pointers, sizes, handlers, outputs): descriptors are validated and
 * staged once and all launch scratch is sized, so rts_plan_launch only
 * enqueues kernels and memsets.  With use_graph != 0 the first launch captures
 * that sequence into a CUDA graph and later launches replay it; Insert, a
 * rebuild or Clear of the index make the next launch re-capture.  Query data
 * and output buffers may be rewritten between launches; their sizes may not.
 * A plan must be destroyed before its index. */
typedef struct rts_plan rts_plan;
int rts_plan_create(rts_index* index, const rts_batch* batches, uint32_t n_batches,
                    rts_plan** out);
int rts_plan_launch(rts_plan* plan, void* stream, int use_graph);
int rts_plan_destroy(rts_plan* plan);

/* Refit-vs-rebuild tuner (no counterpart in the reference, which always
 * refits the touched GASes, spatial_index.cuh:237-264).  Report the duration
 * of the query work that runs between updates (e.g. one round); the library
 * models it as t0 * (1 + a * f), f = fraction of boxes updated since the last
 * re-sort, times its own re-sorts (R), and sets rebuild_update_fraction to
 * sqrt(2 R u / (t0 a)) (u = updated fraction per report), the value that
 * minimises re-sort cost plus expected query slowdown.  The new threshold is
 * returned in *rebuild_update_fraction (nullable). */
int rts_report_query_time(rts_index* index, double query_ms, float* rebuild_update_fraction);

/* ---- autotuner ----------------------------------------------------------------
 * No counterpart in the reference (its only tuning is the intersects
 * parallelism cost model, spatial_index.cuh:690-760, which does not exist
 * here).  Times candidate launch settings — traversal scheme, register cap,
 * curve-ordered visiting, chunk size and, with tune_width, the node width
 * (= leaf size) — on the given batches and keeps the fastest in the index.
 * The batches run through the tuner's own counters and queues: their handlers
 * and outputs are not touched.  With tune_width the index is re-sorted at
 * each candidate width and left at the fastest (its sub-trees merge into
 * one).  Synchronous. */
typedef struct rts_tune_result {
  int32_t node_width, traversal, query_occupancy, sort_queries;
  uint32_t chunk, candidates;
  int32_t collecting; /* 1: timed with the collecting handler, 0: counting (huge results) */
  int32_t group_loads; /* RTS_LOADS_CACHED or RTS_LOADS_STREAMING, as kept */
  double best_ms;     /* median launch time of the kept settings */
  double first_ms;    /* median launch time of the first candidate */
} rts_tune_result;
int rts_autotune(rts_index* index, const rts_batch* batches, uint32_t n_batches, int tune_width,
                 void* stream, rts_tune_result* out);

/* ---- serving engine ---------------------------------------------------------
 * No counterpart in the reference (its Query is a blocking-free launch per
 * call with no admission or batching).  A server owns an index while it
 * exists and serves requests from any host thread in submission order:
 * query requests (host arrays of any size) are cut into parts and packed
 * into persistent launches, several launches in flight on their own streams;
 * a part is admitted while its launch's device arena has room for its queries
 * and estimated pairs.  Update requests (deletes, inserts, updates) apply
 * after every query submitted before them and before every later one.  A
 * request's pairs carry its own 0-based query ids and equal those of the same
 * query made alone on the index state it was submitted against.  A double
 * index is served with the _F64 query kinds. */
typedef struct rts_server rts_server;
typedef struct rts_server_config {
  uint32_t slots;                  /* launches in flight (1..8) */
  uint32_t max_parts_per_launch;   /* request parts per launch */
  uint64_t max_queries_per_launch; /* query capacity of one launch arena */
  uint64_t pairs_per_launch;       /* pair capacity of one launch arena */
  uint64_t hbm_budget_bytes;       /* bound on all arenas (0 = half the free HBM) */
  uint64_t host_result_bytes;      /* pinned host memory holding results until taken */
  uint32_t use_graphs;             /* 1 (default): each launch replays its slot's CUDA graph of
                                      the sequence (input copies, order sort, kernel, count copy),
                                      updated in place; 0: direct launches */
  uint32_t reserved;
} rts_server_config;
typedef struct rts_server_stats {
  uint64_t requests_done, queries_done, pairs_done, launches, retried_parts, updates_done;
  double latency_p50_s, latency_p99_s, latency_max_s; /* submit -> results on the host */
  double elapsed_s;                                   /* first submit -> last completion */
  /* Where the time went, summed over launches since the last reset: */
  double pack_s;    /* worker thread: packing parts into pinned staging */
  double launch_s;  /* device: a launch's query copy, sort, kernel and count copy */
  double copy_s;    /* device: copies of pairs into the pinned result arena */
  double take_s;    /* client threads: rts_server_take copying pairs out */
  double update_s;  /* worker thread: applying update batches (waits for their device work) */
  uint64_t parts;   /* request parts launched */
  uint64_t graph_launches;  /* launches that replayed their slot's CUDA graph */
  double issue_s;   /* worker thread: issuing launches (API calls, or capture + update + replay) */
} rts_server_stats;
int rts_server_config_default(rts_server_config* cfg);
/* Creating a server reserves the index's update capacity (twice its used
 * slots and ids, and the buffers of a full re-sort) so that update batches
 * allocate nothing on the request path. */
int rts_server_create(rts_index* index, const rts_server_config* cfg, rts_server** out);
/* Finishes every submitted request, then stops. */
int rts_server_destroy(rts_server* server);
/* Copies the n queries (points: 2 floats, envelopes: 4) and returns a ticket. */
int rts_server_submit_query(rts_server* server, int query_kind, int predicate,
                            const float* queries, uint64_t n, uint64_t* ticket);
/* Copies an update batch: deletes, then updates, then inserts (new ids are
 * handed out in submission order; rts_server_take reports the first one).
 * A double index (coord_bits = 64) takes deletes only here. */
int rts_server_submit_update(rts_server* server, const uint64_t* delete_ids, uint64_t n_delete,
                             const float* insert_envelopes, uint64_t n_insert,
                             const rts_update_entry* updates, uint64_t n_update,
                             uint64_t* ticket);
/* Waits until the request is done (timeout < 0: no limit); RTS_ERR_TIMEOUT. */
int rts_server_wait(rts_server* server, uint64_t ticket, double timeout_s);
/* Copies a done query's pairs (RTS_ERR_QUEUE_FULL with *n_pairs set when
 * capacity is too small) and forgets the ticket.  For an update ticket,
 * *n_pairs = the first id its inserts received. */
int rts_server_take(rts_server* server, uint64_t ticket, rts_pair* out, uint64_t capacity,
                    uint64_t* n_pairs);
/* Zero-copy access to a done query's pairs: the pinned host segments that
 * hold them, in query order of the request's parts (up to max_segments;
 * *n_segments gives the number needed, RTS_ERR_QUEUE_FULL when larger), and
 * their total.  The memory stays valid, and the ticket reserved, until
 * rts_server_release(ticket). */
int rts_server_view(rts_server* server, uint64_t ticket, const rts_pair** segments,
                    uint64_t* segment_pairs, uint32_t max_segments, uint32_t* n_segments,
                    uint64_t* n_pairs);
/* Returns a viewed request's pinned memory to the server and forgets it. */
int rts_server_release(rts_server* server, uint64_t ticket);
int rts_server_get_stats(rts_server* server, rts_server_stats* stats);
int rts_server_reset_stats(rts_server* server);

/* No counterpart in the reference.  The same arguments, checks and results
 * as rts_query_batched (float and _F64 query kinds, the same traversal
 * scheme), but it allocates no memory: for callers that cannot call
 * cudaMalloc once they are serving (HBM reserved up front, allocation
 * forbidden on the request path, buffers only from the host engine's own
 * memory manager).  Its scratch — the device work counter and the device copy
 * of the batch descriptors — is a fixed array in the library (about 49 KB per
 * device that loads it, held until the process exits) instead of index-owned
 * buffers.  Queries are visited in the order given: the curve-order sort of
 * rts_query_batched needs scratch the size of the launch, so this call skips
 * it (same pairs, possibly slower on large unsorted batches).  At most
 * RTS_NOALLOC_MAX_BATCHES non-empty batches per call (RTS_ERR_CAPACITY
 * otherwise; empty batches do not count).  All calls on a device share that
 * array: calls that overlap on the GPU race.  The first call on a device looks
 * up the array's device address.  The index must already be built; inputs and outputs are the caller's, as in
 * rts_query_batched. */
#define RTS_NOALLOC_MAX_BATCHES 1024
int rts_query_batched_noalloc(rts_index* index, const rts_batch* batches, uint32_t n_batches,
                              void* stream);

/* ---- handler modules ------------------------------------------------------
 * Replaces the reference's shader build with the user's handler header
 * (RTSPATIAL_COMPILE_SHADERS, CMakeLists.txt:73-104) and the PTX modules that
 * SpatialIndex::Init loads from Config::ptx_root (spatial_index.cuh:83-87).
 * The module is a cubin compiled from rtspatial_b200/shaders/
 * rts_handler_module.cu with the handler header force-included
 * (cmake/rtspatial_shaders.cmake, or python -m rtspatial_b200.handlers).  Loading
 * it lets the index's queries take RTS_HANDLER_MODULE: the module's kernels
 * walk the same tree and call rtspatial_handle_* once per pair.  A module built
 * from the shipped counting or collecting header runs this library's own
 * warp-aggregated handler of that behaviour instead (same results).  Loading
 * another module replaces the previous one; the module stays loaded until the
 * index is destroyed.  RTS_ERR_INVALID_ARGUMENT when the file is not a handler
 * module of this library's version (its error names what was missing). */
int rts_load_handler_module(rts_index* index, const char* cubin_path);
/* The built-in handler a loaded module stands for (RTS_HANDLER_COUNT or
 * RTS_HANDLER_COLLECT), or -1 when it calls the user's own functions or no
 * module is loaded. */
int rts_handler_module_builtin(const rts_index* index);

/* ---- introspection ------------------------------------------------------ */
uint64_t rts_size(const rts_index* index);       /* number of ids handed out */
uint32_t rts_num_trees(const rts_index* index);  /* sub-trees currently indexed */
/* Device bytes held by the index (SpatialIndex::PrintMemoryUsage,
 * spatial_index.cuh:893-903). */
uint64_t rts_memory_usage(const rts_index* index);
/* No counterpart in the reference.  Waits for `stream` and reads the index's
 * device status word: bits that query kernels set when they stopped early
 * instead of spinning on (bit 0: a bounded wait for a shared-memory bulk copy
 * of the staged scheme ran out; the launch's results are then incomplete).
 * 0 after every launch that completed normally.  The bits stay set. */
#define RTS_STATUS_WAIT_TIMEOUT 1u
int rts_device_status(rts_index* index, uint32_t* status, void* stream);
/* No counterpart in the reference.  The library's device memory on `device`
 * (an ordinal): every device buffer of every index, plan and server comes
 * from the library's caching allocator, which keeps freed blocks for reuse
 * (stream-ordered: a block freed on one stream and reused on another is
 * waited for).  `reserved` = bytes held from cudaMalloc, `used` = bytes in
 * live buffers; both 0 before the library's first allocation there. */
int rts_memory_pool_stats(int device, uint64_t* reserved, uint64_t* used);
/* Returns the kept, unused blocks on `device` to the driver, after a
 * synchronisation of that device (rts_destroy does this too). */
int rts_trim_memory(int device);
/* Message of the last failing call on this thread ("" if none). */
const char* rts_last_error(void);
/* Library version string. */
const char* rts_version(void);

#ifdef __cplusplus
}
#endif

#endif /* RTSPATIAL_B200_H */
