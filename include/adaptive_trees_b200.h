/* adaptive_trees_b200.h -- C ABI of the B200 adaptive-tree engine.
 *
 * Plain C: handles, pointers, sizes and status codes; no C++ or framework
 * types.  Each entry point replaces one member of the reference's C++ surface
 * (nrottstegge/Adaptive_Trees, include/adaptive_octree/tree.hpp), cited at
 * the declaration.  Coordinates and returned buffers are DEVICE pointers; the
 * stream is a cudaStream_t passed as void* (NULL = legacy default stream).
 *
 * Error behaviour: the reference throws std::invalid_argument,
 * std::logic_error and std::length_error from its C++ API and calls
 * std::exit() on CUDA errors.  Here every entry point returns an ao_status;
 * ao_last_error() returns the message of the last failure on the calling
 * thread.  Nothing in the library exits the process.
 */
#ifndef ADAPTIVE_TREES_B200_H
#define ADAPTIVE_TREES_B200_H

#include <stddef.h>

#if defined(__GNUC__)
#define AO_API __attribute__((visibility("default")))
#else
#define AO_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef enum ao_status
{
    AO_OK = 0,
    AO_ERR_INVALID_ARGUMENT = 1, /* std::invalid_argument in the reference */
    AO_ERR_LOGIC = 2,            /* std::logic_error (wrong call order, unsupported getter) */
    AO_ERR_LENGTH = 3,           /* std::length_error (capacity beyond the node index range) */
    AO_ERR_CUDA = 4,             /* CUDA runtime failure (the reference exits the process) */
    AO_ERR_OUT_OF_MEMORY = 5,    /* device or host allocation failed */
    AO_ERR_RUNTIME = 6           /* other failure, e.g. a bounded device wait gave up */
} ao_status;

enum { AO_OCTREE = 0, AO_BINARY = 1 };          /* TreeType (config.hpp:50) */
enum { AO_FLOAT32 = 0, AO_FLOAT64 = 1 };        /* Real */
enum { AO_LEAF_COUNT = 0, AO_NF_COUNT = 1 };    /* SplitCriterion (config.hpp:51) */
enum { AO_MORTON = 0, AO_HILBERT = 1 };         /* SfcKind (config.hpp:52) */

/* Getter selectors: the reference's device_vector getters (tree.hpp:72-97, 113). */
enum
{
    AO_BUF_PARTICLE_KEYS = 0,        /* particleKeys_d      u64, numParticles             */
    AO_BUF_PERM = 1,                 /* perm_d              u32, numParticles             */
    AO_BUF_CORNERSTONE = 2,          /* cornerstone_d       u64, numLeaves + 1            */
    AO_BUF_LEAF_COUNTS = 3,          /* leafCounts_d        u32, numLeaves                */
    AO_BUF_NEAR_FIELD_COUNTS = 4,    /* nearFieldCounts_d   u32, numLeaves (octree only)  */
    AO_BUF_SFC_BOX_INDEX = 5,        /* sfcBoxIndex_d       u64, numNodes                 */
    AO_BUF_HAS_BOX_SPLIT = 6,        /* hasBoxSplit_d       u8,  numNodes                 */
    AO_BUF_BOX_DEPTH = 7,            /* boxDepth_d          u8,  numNodes                 */
    AO_BUF_PARENT_INDEX = 8,         /* parentIndex_d       i32, numNodes                 */
    AO_BUF_CHILD_INDEX = 9,          /* childIndex_d        i32, numNodes                 */
    AO_BUF_LEVEL_OFFSET = 10,        /* levelOffset_d       i32, 23 (octree) / 65 (binary) */
    AO_BUF_PARTICLE_BEGIN_INDEX = 11,/* particleBeginIndex_d u32, numNodes                */
    AO_BUF_PARTICLE_COUNTS = 12,     /* particleCounts_d    u32, numNodes + 1             */
    AO_BUF_SFC_PARTICLE_INDEX = 13,  /* sfcParticleIndex_d  u64, numActiveParticles       */
    AO_BUF_LEAF_BEGINS = 14          /* first particle (index into P) of every leaf and the active end,
                                        u32, numLeaves + 1; no getter in the reference (its counts'
                                        prefix sum), kept by this engine for the near field of an FMM */
};

/* TreeConfig<Real> (config.hpp:147-160); the box is given in double and
 * converted to Real. */
typedef struct ao_config
{
    int max_depth;                   /* -1: backend default (21 octree build rounds / 63 binary depth) */
    unsigned max_particles_per_leaf; /* LeafCount bucket, or the near-field limit for NFCount */
    int update_iterations;           /* -1: backend default (2 octree / 6 binary) */
    double box[6];                   /* xmin, xmax, ymin, ymax, zmin, zmax */
    int split_criterion;             /* AO_LEAF_COUNT / AO_NF_COUNT */
    int sfc_kind;                    /* AO_MORTON / AO_HILBERT */
    int views_tree_structure;        /* ViewConfig (config.hpp:115-120) */
    int views_particle_counts;
    int views_particle_mapping;
} ao_config;

typedef struct ao_view_config
{
    int tree_structure;
    int particle_counts_per_box;
    int particle_mapping;
} ao_view_config;

typedef struct ao_tree_info
{
    size_t num_particles;        /* numParticles()        tree.hpp:64-65 */
    size_t num_active_particles; /* numActiveParticles()  tree.hpp:66-67 */
    size_t num_nodes;            /* numNodes()            tree.hpp:68-69 */
    size_t num_leaves;           /* cornerstone_d().size() - 1 */
    size_t leaf_capacity;        /* capacity that bounds update() before needsResize */
    unsigned max_achieved_depth; /* maxAchievedDepth()    tree.hpp:70-71 */
    int split_criterion;         /* splitCriterion()      tree.hpp:99-103 */
    int sfc_kind;                /* sfcKind() tree.hpp:104-108; -1 for Binary (the C++ facade throws) */
    unsigned long long kernel_launches; /* engine kernels launched by this process so far */
} ao_tree_info;

typedef struct ao_tree ao_tree;

/* Tree<Real, Kind>::Tree(x, y, z, count, config) -- tree.hpp:35-37 (with the
 * backend constructors octree.cu:321-416, kdtree3d.cu:175-216).  x, y, z are
 * borrowed device arrays of `n` Real values; they are read at every build()
 * and update() and may be changed in place between calls. */
AO_API ao_status ao_tree_create(int kind, int real_type, const void *x, const void *y, const void *z, size_t n,
                         const ao_config *config, void *stream, ao_tree **out);

/* ~Tree() */
AO_API ao_status ao_tree_destroy(ao_tree *tree);

/* Tree::build() -- tree.hpp:45 (octree.cu:427-469, kdtree3d.cu:227-257).  Not capturable. */
AO_API ao_status ao_tree_build(ao_tree *tree);

/* Tree::update() -- tree.hpp:46 (octree.cu:471-481, kdtree3d.cu:259-270).
 * Capturable into a CUDA graph on the tree's stream. */
AO_API ao_status ao_tree_update(ao_tree *tree);

/* Stage timing of build() and update(): the CUDA-event counterpart of the
 * reference's NVTX ranges behind ADAPTIVE_OCTREE_PROFILING (config.hpp:20-28,
 * octree.cu:287-306).  With profiling on, each octree build() and update()
 * not made under stream capture records events at its stage boundaries and
 * around every near-field launch on the tree's stream, and pushes one NVTX
 * range per stage. */
typedef struct ao_stage_times {
    double keys_and_sort_ms; /* key generation, the 8 sort passes and the key sample */
    double refresh_ms;       /* update: the full per-leaf refresh (begin indices, cell table, near field) */
    double passes_ms;        /* the rebalance passes (build: its rounds, with the host's checks between them) */
    double finish_ms;        /* leaf counts and views (build: and the final copies) */
    double total_ms;
    double near_field_ms;    /* all near-field kernel launches of the call (0 without NFCount) */
    double near_field_first_ms; /* the first of them (update(): the full refresh of every leaf) */
    int near_field_launches;
    int call;                /* 1 build, 2 update */
    int valid;               /* 0: no profiled call since profiling was switched on */
} ao_stage_times;
AO_API ao_status ao_tree_set_profiling(ao_tree *tree, int on);
/* Waits for the last profiled build() or update() and reads its stage times. */
AO_API ao_status ao_tree_stage_times(ao_tree *tree, ao_stage_times *out);

/* How an octree build() reaches its tree (no counterpart in the reference,
 * whose build runs split/merge rounds until one changes nothing,
 * octree.cu:159-180).  Mode 0 (default) builds the converged tree directly,
 * one level of internal nodes at a time, and derives from the same cells how
 * many leaves each of the reference's rounds would have held (the capacity
 * history behind leafCapacity); it falls back to the rounds when the tree
 * would not converge within max_depth rounds or when LeafCount's 32-bit split
 * thresholds wrap (bucket >= 2^23).  Mode 1 always runs the rounds.  Both
 * give the same tree, counts and capacity.  Binary (k-d) trees likewise:
 * mode 0 builds the converged tree a depth at a time (the reference's build
 * passes, kdtree3d.cu:239-249, split one depth per pass), falling back to
 * the passes for a max_depth above 63; mode 1 always runs the passes. */
AO_API ao_status ao_tree_set_build_mode(ao_tree *tree, int mode);
/* The last build(): *by_levels = 1 when it used the level builder; *rounds =
 * the build rounds that changed the tree (the reference's history length).
 * Either pointer may be NULL. */
AO_API ao_status ao_tree_build_path(ao_tree *tree, int *by_levels, int *rounds);

/* Opt-in extension with no reference counterpart: update() that keeps
 * passing until a pass changes nothing or would exceed the leaf capacity
 * (then doBuffersNeedResize() reports it, as after update()), at most
 * max_passes (>= 1).  The reference's update() runs a fixed pass count
 * (octree.cu:471-481, kdtree3d.cu:259-270), which can leave overfull or
 * mergeable leaves on fast-moving particles.  The tree equals update() with
 * update_iterations = max_passes.  Reads the device state between groups of
 * update_iterations passes, so it is not capturable.  changed_passes (may be
 * NULL; setting it adds one host wait) receives the passes that changed the
 * tree. */
AO_API ao_status ao_tree_update_until_converged(ao_tree *tree, int max_passes, int *changed_passes);

/* Tree::computeViews() / computeViews(ViewConfig) -- tree.hpp:49-53.
 * views == NULL uses the configured views. */
AO_API ao_status ao_tree_compute_views(ao_tree *tree, const ao_view_config *views);

/* Tree::doBuffersNeedResize() -- tree.hpp:56-57.  Refreshes the host-visible
 * sizes from the device state; *out = 1 when resizeBuffers() is needed. */
AO_API ao_status ao_tree_needs_resize(ao_tree *tree, int *out);

/* Tree::resizeBuffers() -- tree.hpp:47.  Grows the leaf capacity by 25%;
 * graphs captured before must be captured again. */
AO_API ao_status ao_tree_resize_buffers(ao_tree *tree);

/* Getters particleKeys_d() ... sfcParticleIndex_d() -- tree.hpp:72-97, 113:
 * device pointer, logical length (elements) and allocated capacity. */
AO_API ao_status ao_tree_get_buffer(ao_tree *tree, int which, const void **dptr, size_t *len, size_t *capacity);

/* numLeaves_d() / numNodes_d() / numActiveParticles_d() -- tree.hpp:58-63:
 * device-resident counters for kernels recorded in the same graph. */
AO_API ao_status ao_tree_counters(ao_tree *tree, const int **num_leaves_d, const int **num_nodes_d,
                           const unsigned **num_active_particles_d);

/* numParticles(), numActiveParticles(), numNodes(), maxAchievedDepth(),
 * splitCriterion(), sfcKind() -- tree.hpp:64-71, 99-108. */
AO_API ao_status ao_tree_get_info(ao_tree *tree, ao_tree_info *info);

/* computeSfcKeys (sfc_keys.cuh:517-532) / computeSfcKeysBinary
 * (kdtree3d_rebalance.cuh:261-273): unsorted keys of n particles and, if
 * perm_d is not NULL, the identity permutation.  kind AO_OCTREE uses
 * sfc_kind; AO_BINARY uses the longest-side schedule of `box` and max_depth. */
AO_API ao_status ao_compute_sfc_keys(int kind, int real_type, const void *x, const void *y, const void *z, size_t n,
                              const double *box, int sfc_kind, unsigned max_depth, unsigned long long *keys_d,
                              unsigned *perm_d, void *stream);

/* cub::DeviceRadixSort::SortPairs(d_temp_storage, temp_storage_bytes,
 * d_keys_in, d_keys_out, d_values_in, d_values_out, num_items, begin_bit,
 * end_bit, stream) as called at octree.cu:301-304 and kdtree3d.cu:168-170:
 * stable LSD sort of 64-bit keys carrying 32-bit values by bits
 * [begin_bit, end_bit), onesweep with decoupled look-back.  With scratch ==
 * NULL only *scratch_bytes is set.  values_in == NULL sorts the indices
 * 0..n-1 (the identity permutation).  keys_in/values_in are not modified and
 * must not alias the outputs.  No allocation; capturable.  The sort uses
 * the configuration the sort tuner holds for n (below); the size query
 * answers for the largest configuration, so the scratch fits any of them. */
AO_API ao_status ao_sort_pairs(void *scratch, size_t *scratch_bytes, const unsigned long long *keys_in,
                               unsigned long long *keys_out, const unsigned *values_in, unsigned *values_out,
                               size_t n, int begin_bit, int end_bit, void *stream);

/* Waits for `stream` and checks the last ao_sort_pairs of n items that ran
 * in `scratch`: AO_ERR_RUNTIME when a look-back wait of the sort gave up
 * after its bounded number of polls (the output is then not sorted; CUB's
 * SortPairs has no such failure, its waits are unbounded), AO_OK otherwise.
 * No counterpart in the reference.  n = 0 returns AO_OK. */
AO_API ao_status ao_sort_pairs_check(const void *scratch, size_t n, void *stream);

/* Self-test of the bounded device waits (no counterpart in the reference).
 * Runs one look-back -- which 0: a radix sort pass, 1: the rebalance
 * decide+scan -- whose predecessor tile is never processed, so its wait can
 * only end by its limit of spin_limit polls (1..65536).  Returns
 * AO_ERR_RUNTIME with *error_word (may be NULL) set to the kernel's error
 * code when the wait gave up and the kernel returned, the designed outcome;
 * the device stays usable.  Uses its own small allocations and stream. */
AO_API ao_status ao_selftest_bounded_wait(int which, unsigned spin_limit, int *error_word);

/* The sort tuner (no counterpart in the reference; it picks what the
 * reference leaves to CUB's fixed policy).  The radix sort is compiled in a
 * few configurations of digit width (7 or 8 bits) and keys per thread (8 to
 * 16; a tile is 256 threads times that).  The first octree or forest build
 * of a size class (sizes grouped by bit length) on a device times every
 * configuration on its own keys and keeps the fastest for that device, size
 * class and kind (contiguous: trees and ao_sort_pairs; segmented: batches).
 * Every configuration gives the same sorted output. */
AO_API ao_status ao_sort_config_count(int *count);
AO_API ao_status ao_sort_config_info(int config, int *digit_bits, int *items_per_thread);
/* The configuration the next sort of n keys uses on the current device;
 * *tuned = 1 when it was chosen by timing. */
AO_API ao_status ao_sort_tuning(int segmented, size_t n, int *config, int *digit_bits, int *items_per_thread,
                                int *tuned);
/* on = 0: no timing; untuned sizes use the default configuration. */
AO_API ao_status ao_sort_set_autotune(int on);
/* Every sort uses `config` (-1 lifts this). */
AO_API ao_status ao_sort_force_config(int config);
/* Forgets the tuned choices of every device. */
AO_API ao_status ao_sort_forget_tuning(void);

/* Allocation-free variant of ao_sort_pairs; it has no counterpart in the
 * reference.  The same sort, with its scratch in a fixed device array inside
 * this library instead of caller memory, for callers that cannot allocate
 * device memory where they sort: a process that reserves its whole device
 * budget at start-up and must not grow it, or a plain C / FFI host without a
 * device allocator of its own.
 *  - n <= AO_SORT_PAIRS_NOALLOC_MAX_ITEMS, else AO_ERR_INVALID_ARGUMENT.
 *  - The first call on a device does the set-up (it loads every kernel the
 *    sort can launch there); make it before any stream capture.  Every call
 *    looks up the array's address on the current device, so a device whose
 *    context was torn down and created again is handled.
 *  - One array per device: calls that overlap in time on the same device
 *    (other streams, other threads) race and corrupt each other's results.
 *    Serialise them.
 *  - Arguments otherwise as ao_sort_pairs. */
#define AO_SORT_PAIRS_NOALLOC_MAX_ITEMS 1048576
AO_API ao_status ao_sort_pairs_noalloc(const unsigned long long *keys_in, unsigned long long *keys_out,
                                       const unsigned *values_in, unsigned *values_out, size_t n, int begin_bit,
                                       int end_bit, void *stream);
/* Waits for `stream` and checks the last ao_sort_pairs_noalloc of n items on
 * the current device, as ao_sort_pairs_check does for caller scratch. */
AO_API ao_status ao_sort_pairs_noalloc_check(size_t n, void *stream);

/* ---------------------------------------------------------------------------
 * Batched octrees ("forest").  The reference has no batch API: its callers
 * loop over one Tree<Real, Octree> per particle system.  A batch holds many
 * independent systems, each with its own borrowed device coordinates and
 * count, and one shared config (octree, LeafCount, Morton or Hilbert, no
 * views).  Every system gets exactly what a Tree built and updated on that
 * system alone would hold: particleKeys_d, perm_d (indices within the
 * system), cornerstone_d, leafCounts_d, leafCapacity and needsResize.  The
 * work of all systems runs in the same kernel launches (a segmented sort and
 * one decision/scan/scatter per round or pass over all systems' leaves), so
 * many small systems are not bound by launch latency.
 * ------------------------------------------------------------------------- */
typedef struct ao_batch ao_batch;

typedef struct ao_batch_system_info
{
    size_t num_particles;
    size_t num_active_particles;
    size_t num_leaves;
    size_t leaf_capacity;
    int needs_resize;
} ao_batch_system_info;

/* One Tree<Real, Octree>(x[s], y[s], z[s], counts[s], config) per system s
 * (tree.hpp:25), all on `stream`.  AO_ERR_INVALID_ARGUMENT for NFCount, views,
 * a binary kind or more than 2^32 - 1 particles in total. */
AO_API ao_status ao_batch_create(int real_type, int num_systems, const void *const *x, const void *const *y,
                                 const void *const *z, const size_t *counts, const ao_config *config, void *stream,
                                 ao_batch **out);
AO_API ao_status ao_batch_destroy(ao_batch *batch);
/* build() of every system (octree.cu:427-457). */
AO_API ao_status ao_batch_build(ao_batch *batch);
/* Mode 0 (default): build() makes every system's converged tree by levels in
 * one persistent launch after the sort, falling back to the rounds where a
 * system's rounds would not converge within max_depth; mode 1: always the
 * rounds.  Both give the same trees, counts and capacities. */
AO_API ao_status ao_batch_set_build_mode(ao_batch *batch, int mode);
/* *by_levels = 1 when the last build() used the level builder. */
AO_API ao_status ao_batch_build_path(ao_batch *batch, int *by_levels);
/* update() of every system (octree.cu:459-496); capturable when frozen is
 * NULL.  frozen: optional host array of num_systems bytes; a system marked
 * non-zero keeps its tree, as if update() were not called on it (for the
 * resize-and-retry step of the systems that needed a resize). */
AO_API ao_status ao_batch_update(ao_batch *batch, const unsigned char *frozen);
/* Opt-in extension (see ao_tree_update_until_converged): update passes until
 * a pass changes no system, at most max_passes (>= 1); every system's tree
 * equals update() with update_iterations = max_passes.  Not capturable.
 * changed_passes (may be NULL) receives the passes that changed some system. */
AO_API ao_status ao_batch_update_until_converged(ao_batch *batch, const unsigned char *frozen, int max_passes,
                                                 int *changed_passes);
/* doBuffersNeedResize() of every system; *any = 1 if one of them needs it. */
AO_API ao_status ao_batch_needs_resize(ao_batch *batch, int *any);
/* resizeBuffers() of every system that needs a resize. */
AO_API ao_status ao_batch_resize_buffers(ao_batch *batch);
/* New coordinate pointers of one system (same count). */
AO_API ao_status ao_batch_set_coordinates(ao_batch *batch, int system, const void *x, const void *y, const void *z);
/* Getter of one system: AO_BUF_PARTICLE_KEYS, AO_BUF_PERM, AO_BUF_CORNERSTONE
 * or AO_BUF_LEAF_COUNTS; sizes as of the last build/needs_resize. */
AO_API ao_status ao_batch_get_buffer(ao_batch *batch, int system, int which, const void **ptr, size_t *size);
AO_API ao_status ao_batch_get_info(ao_batch *batch, int system, ao_batch_system_info *info);

/* ---------------------------------------------------------------------------
 * Serving.  The reference has no serving layer: its callers build and update
 * trees one at a time.  A server takes requests to build new trees and to
 * update or release resident ones, and runs them on `slots` worker threads:
 * every resident tree keeps its buffers and its own copy of its coordinates
 * on the device between requests and runs on its own stream, so requests on
 * different trees overlap on the GPU.  Builds are admitted in arrival order
 * when their memory fits `memory_budget_bytes` next to the resident trees;
 * updates and releases pass waiting builds; requests on one tree run in
 * arrival order.  An update that exceeds the tree's capacity is completed by
 * resizeBuffers() and another update(), as the reference's callers do.  Each
 * request gives the result it gives when it runs alone.
 * ------------------------------------------------------------------------- */
typedef struct ao_server ao_server;

enum { AO_REQUEST_BUILD = 0, AO_REQUEST_UPDATE = 1, AO_REQUEST_RELEASE = 2 };

typedef struct ao_request
{
    int op;             /* AO_REQUEST_BUILD / _UPDATE / _RELEASE */
    long long tree;     /* caller-chosen id, unique among resident trees */
    int kind;           /* build: AO_OCTREE / AO_BINARY */
    int real_type;      /* build: AO_FLOAT32 / AO_FLOAT64 */
    ao_config config;   /* build */
    size_t n;           /* build: particles; update: the tree's particle count */
    const void *x, *y, *z; /* build/update: coordinates (device or pinned host), copied into the
                            tree's own storage when the request starts: keep them valid and
                            unchanged until the request completes */
    int want_digest;    /* 1: hash the tree's keys, perm, cornerstone and counts when done */
} ao_request;

typedef struct ao_request_result
{
    int status;                /* ao_status of the request */
    double queued_ms;          /* submit -> start */
    double latency_ms;         /* submit -> result ready */
    size_t num_leaves;
    int resizes;               /* resize-and-retry steps of an update */
    unsigned long long digest; /* with want_digest */
} ao_request_result;

typedef struct ao_serve_stats
{
    size_t submitted, completed, failed, resident_trees, resident_bytes, peak_bytes;
    unsigned long long particles; /* particles of the completed builds and updates */
    double p50_ms, p99_ms, mean_ms, max_ms; /* request latency, submit -> result ready */
    double particles_per_s, span_s;         /* over first submit -> last completion */
} ao_serve_stats;

AO_API ao_status ao_serve_create(int slots, size_t memory_budget_bytes, ao_server **out);
/* Requests still queued end with AO_ERR_RUNTIME; running ones complete. */
AO_API ao_status ao_serve_destroy(ao_server *server);
/* Queues a request; returns at once. */
AO_API ao_status ao_serve_submit(ao_server *server, const ao_request *request, long long *ticket);
/* Blocks until the request is done; returns its status (message in ao_last_error). */
AO_API ao_status ao_serve_wait(ao_server *server, long long ticket, ao_request_result *result);
/* Blocks until every submitted request is done. */
AO_API ao_status ao_serve_drain(ao_server *server);
AO_API ao_status ao_serve_get_stats(ao_server *server, ao_serve_stats *stats);
AO_API ao_status ao_serve_reset_stats(ao_server *server);

/* Freed device blocks are kept for reuse by later trees (cudaMalloc and
 * cudaFree would synchronise the device); this hands them back to the driver. */
AO_API ao_status ao_release_cached_memory(void);

/* Per-particle data in key order, the gather an FMM does after the tree is
 * built (no entry point in the reference; its callers index with perm_d):
 * dst[i] = src[perm[i]] for the tree's numParticles() elements of
 * elem_bytes each.  Device pointers, not overlapping; on the tree's stream. */
AO_API ao_status ao_tree_gather(ao_tree *tree, const void *src, void *dst, size_t elem_bytes);

/* ---------------------------------------------------------------------------
 * Particle files and dataset manifests of the reference's tests and benchmarks
 * (tests/particle_io.hpp; benchmarks/drivers/common.hpp:62-175), so the same
 * inputs feed this engine.  Text rows: four numbers in charge-x-y-z or
 * x-y-z-charge order, or ESC for an escaped particle that keeps its slot
 * (blank and '#' rows skipped).  Binary frames: x y z doubles, NaN x = escaped.
 * Escaped particles read as the escape coordinate (DBL_MAX) on every axis.
 * ------------------------------------------------------------------------- */
enum { AO_LAYOUT_CHARGE_XYZ = 0, AO_LAYOUT_XYZ_CHARGE = 1, AO_LAYOUT_BINARY_XYZ = 2 };

/* *x, *y, *z receive malloc'ed host arrays of *n doubles; release them with ao_free. */
AO_API ao_status ao_read_particles(const char *path, int layout, double **x, double **y, double **z, size_t *n);
AO_API ao_status ao_free(void *p);

typedef struct ao_manifest ao_manifest;
AO_API ao_status ao_read_manifest(const char *path, ao_manifest **out);
/* dataset name, particle slots of every frame, the shared box, frame count */
AO_API ao_status ao_manifest_info(const ao_manifest *manifest, const char **dataset, size_t *slots, double *box6,
                                  size_t *frames);
/* frame i: its index and id, layout (AO_LAYOUT_*), and file path (relative
 * paths resolved against the manifest's directory) */
AO_API ao_status ao_manifest_frame(const ao_manifest *manifest, size_t i, int *index, long long *id, int *layout,
                                   const char **path);
AO_API ao_status ao_manifest_destroy(ao_manifest *manifest);

/* Message of the last failed call on this thread ("" if none). */
AO_API const char *ao_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* ADAPTIVE_TREES_B200_H */
