/*
 * cellato_b200.h -- C ABI of the B200 bit-plane hot path.
 *
 * The reference binds this path through C++ class templates (the grid,
 * evaluator and traverser types picked by
 * include/experiments/test_suites.hpp:115-225).  These entry points replace the
 * device side of those templates behind plain pointers and sizes; the C++
 * header shims in 2026-cellato-smpt-journal_b200/include/ (memory/,
 * traversers/cuda/) call them so that the reference's callers compile
 * unchanged.  Every function returns a cellato_status; none allocates unless
 * its name says so, none frees caller memory, and all work is ordered on the
 * given CUDA stream (0 = legacy default stream).
 *
 * Cells and layouts.  A grid of X x Y cells of an automaton with nb = needed
 * bits is nb *planes*; plane i holds bit i of every cell's state-dictionary
 * index.  Plane bytes are exactly the reference's:
 *   CELLATO_LAYOUT_BIT_PLANES        include/memory/bit_planes_grid.hpp:234-270
 *     words of W bits, word (x/W, y), bit x%W, least significant = leftmost;
 *   CELLATO_LAYOUT_TILED_BIT_PLANES  include/memory/tiled_bit_planes_grid.hpp:243-288
 *     words of 8 x (W/8) cells, bit (y%(W/8))*8 + x%8, tiles row-major.
 * Each plane is X*Y/8 bytes, 16-byte aligned.  Accepted sizes: X a multiple of
 * 32 (of 64 for W = 64 linear), Y >= 1 (a multiple of W/8 for tiled layouts).
 * The reference's CUDA traversers accept a subset of these (they also need the
 * word counts to divide the CUDA block and temporal tile,
 * include/traversers/cuda/simple.hpp:45-49, temporal.hpp:60-86).
 *
 * Time.  Steps are numbered globally from t0; the parity of each step's number
 * drives alternate_algorithms and the Margolus block phase exactly as the
 * reference's time_step does (include/evaluators/standard.hpp:150-205).
 */
#ifndef CELLATO_B200_H
#define CELLATO_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st* cellato_stream_t; /* == cudaStream_t */

typedef enum {
    CELLATO_OK = 0,
    CELLATO_EINVAL = 1,        /* bad argument (null pointer, unknown id, ...) */
    CELLATO_EINVAL_DIMS = 2,   /* grid sizes not accepted by the layout */
    CELLATO_ESMEM = 3,         /* temporal tile does not fit in shared memory */
    CELLATO_ECUDA = 4,         /* a CUDA runtime call failed; see cellato_last_error() */
    CELLATO_ETIMEDOUT = 5,     /* a bounded device-side wait gave up */
    CELLATO_ENOMEM = 6,        /* allocation failed */
    CELLATO_EUNSUPPORTED = 7   /* combination not built */
} cellato_status;

typedef enum {
    CELLATO_LAYOUT_BIT_PLANES = 0,
    CELLATO_LAYOUT_TILED_BIT_PLANES = 1
} cellato_layout;

/* Rule ids of the ten automata of the reference (src/<automaton>/config.hpp),
 * built into the library.  Rules registered with cellato_rule_register get
 * the ids that follow (CELLATO_BUILTIN_RULES, CELLATO_BUILTIN_RULES + 1, ...). */
typedef enum {
    CELLATO_GAME_OF_LIFE = 0,
    CELLATO_FOREST_FIRE = 1,
    CELLATO_WIRE = 2,
    CELLATO_EXCITABLE = 3,
    CELLATO_BRIAN = 4,
    CELLATO_MAZE = 5,
    CELLATO_CYCLIC = 6,
    CELLATO_FLUID = 7,
    CELLATO_CRITTERS = 8,
    CELLATO_TRAFFIC = 9,
    CELLATO_BUILTIN_RULES = 10
} cellato_rule;

/* Capacity of the rule table: the built-in rules plus registered ones. */
#define CELLATO_MAX_RULES 256

/* Kernel table of one rule (opaque to C).  A C++ translation unit compiled
 * with nvcc for sm_100a builds one for any rule written in the rule DSL with
 * cellato::b200::custom_rule_ops<Config>() (2026-cellato-smpt-journal_b200/
 * include/b200/custom_rule.cuh); the library runs it through every entry point
 * once it is registered. */
typedef struct cellato_rule_ops_st cellato_rule_ops;

/* Per-call tuning of the traversers; NULL or all-zero fields = the library's
 * choices.  The reference passes the same kind of knobs per run in run_params
 * (include/experiments/run_params.hpp:10-43: cuda_block_size_y,
 * temporal_tile_size_y); here they select among this library's kernels.  Every
 * choice gives the same results. */
typedef struct {
    int simple_kernel;   /* single-step kernel: 0 automatic, 1 register bands, 2 bulk-copy streaming (linear
                            layout, rows of 16-byte multiples; others use 1), 3 TMA-fed shared-memory tiles
                            (rows of a multiple of its strip, 4096 cells at one word per lane and 8192 at
                            two or four; others use 1) */
    int row_loop;        /* temporal row loop: 0 automatic, 1 row by row, 2 the input rows of each three-row
                            trip read before its in-place writes, 3 as 2 with two steps per sweep of the
                            tile (an odd last step runs alone) */
    int words_per_lane;  /* words per lane, 0 the default, else 1, 2 or 4.  Temporal tile width: default 2 for
                            one-plane rules, else 1; 2 and 4 only for rules of up to three planes (others use
                            1, and 4 means 2); the tile is 32 x this many words.  TMA single-step kernel: 2 for
                            rules of up to three planes, 4 for one-plane rules outside the 8-row tiled
                            layout; a width the rule or the grid does not allow falls back to the register
                            kernel */
    int tile_rows;       /* temporal tile rows including both k-row halos; 0 the library's default */
} cellato_tune;

/* ---- identity ----------------------------------------------------------- */

/* Library version string, e.g. "cellato-b200 1.0 sm_100a". */
const char* cellato_version(void);

/* Message of the last failing call on this host thread ("" if none). */
const char* cellato_last_error(void);

/* Rule id of a CLI automaton name ("game-of-life", "fire" or "forest-fire",
 * ...; src/main.cpp:55-77) or of a registered rule's name, or -1. */
int cellato_rule_from_name(const char* name);

/* Name of a rule id (the config's `name`, e.g. "forest-fire"), or NULL. */
const char* cellato_rule_name(int rule);

/* needed_bits of the rule's state dictionary (state_dictionary.hpp:22), or -1. */
int cellato_rule_planes(int rule);

/* number_of_values of the rule's state dictionary, or -1. */
int cellato_rule_states(int rule);

/* Number of rule ids in use: CELLATO_BUILTIN_RULES plus the registered rules. */
int cellato_rule_count(void);

/* Adds a rule to the library's rule table and returns its id in *rule_out
 * (the next free id).  `ops` must stay valid until the process exits (the
 * table custom_rule_ops returns does).  CELLATO_EINVAL for a table built
 * against another layout of cellato_rule_ops, a name already in use or a full
 * table.  Registering the same table twice returns its first id.  Thread-safe;
 * ids are never reused.  Replaces the reference's per-automaton explicit
 * instantiation in src/_shared/cuda_instantiation_template.cuh:77-193. */
int cellato_rule_register(const cellato_rule_ops* ops, int* rule_out);

/* Bytes of one plane of an X x Y grid (X*Y/8). */
size_t cellato_plane_bytes(int x_cells, int y_cells);

/* CELLATO_OK if (layout, word_bits, X, Y) is a grid shape this library runs. */
int cellato_check_dims(int layout, int word_bits, int x_cells, int y_cells);

/* ---- plane memory (replaces bit_planes_grid::to_cuda / to_cpu /
 *      free_cuda_memory, bit_planes_grid.hpp:86-95, :132-168; same for the
 *      tiled grid, tiled_bit_planes_grid.hpp:89-98, :141-177) ------------- */

/* cudaMalloc nb planes of `bytes` each into planes_out[0..nb). */
int cellato_planes_alloc(int nb, size_t bytes, void** planes_out);
/* cudaFree nb planes (NULL entries are skipped) and clear the pointers. */
int cellato_planes_free(int nb, void** planes);
/* Stream-ordered copies of nb planes host -> device / device -> host. */
int cellato_planes_upload(int nb, void* const* dev_planes, const void* const* host_planes, size_t bytes,
                          cellato_stream_t stream);
int cellato_planes_download(int nb, void* const* host_planes, const void* const* dev_planes, size_t bytes,
                            cellato_stream_t stream);

/* ---- device packing (replaces the host loops of the grid classes:
 *      bit_planes_grid.hpp:234-270 pack, :97-124 get_cell; tiled
 *      tiled_bit_planes_grid.hpp:243-288, :100-139) ------------------------ */

/* cells: device array of X*Y uint8 state-dictionary indices (row-major);
 * planes: nb device planes in the given layout.  Stream-ordered, no allocation. */
int cellato_pack_cells(int layout, int word_bits, int nb, const uint8_t* cells, int x_cells, int y_cells,
                       void* const* planes, cellato_stream_t stream);
int cellato_unpack_cells(int layout, int word_bits, int nb, const void* const* planes, int x_cells, int y_cells,
                         uint8_t* cells, cellato_stream_t stream);

/* ---- traversers ----------------------------------------------------------- */

/* Simple traverser (replaces include/traversers/cuda/simple.cu:43-87 with
 * process_grid_kernel_simple :20-39): `steps` single-step launches, ping-pong
 * between planes_a (input) and planes_b.  *result_in_b is set to 1 when the
 * final state is in planes_b (odd number of launches), else 0.  tune: NULL or
 * its simple_kernel and words_per_lane fields (the others are ignored).
 * Nothing is allocated; planes_a and planes_b must not overlap. */
int cellato_run_simple(int rule, int layout, int word_bits, void* const* planes_a, void* const* planes_b,
                       int x_cells, int y_cells, int t0, int steps, const cellato_tune* tune,
                       cellato_stream_t stream, int* result_in_b);

/* Temporal traverser (replaces include/traversers/cuda/temporal.cu:137-272
 * with process_grid_kernel_linear_temporal :35-135): launches of k fused steps
 * each (the last launch takes the remainder), ping-pong as above.  k in 1..32.
 * tune: NULL or its row_loop, words_per_lane and tile_rows fields.  Returns
 * CELLATO_ESMEM when the tile does not fit ("temporal tile is too large" in
 * the reference, temporal.cu:214-216). */
int cellato_run_temporal(int rule, int layout, int word_bits, void* const* planes_a, void* const* planes_b,
                         int x_cells, int y_cells, int t0, int steps, int k, const cellato_tune* tune,
                         cellato_stream_t stream, int* result_in_b);

/* Reads and clears the number of bounded device-side waits (mbarrier waits of
 * the streaming single-step kernel) that gave up since the last call; returns
 * CELLATO_ETIMEDOUT when it is non-zero.  Synchronises the device.  No
 * counterpart in the reference, whose kernels never wait. */
int cellato_device_wait_timeouts(unsigned* count);

/* ---- batches: many independent grids per launch -------------------------
 * No counterpart in the reference (one grid per traverser run).  Results are
 * identical to cellato_run_temporal on each grid alone with the same k. */

typedef struct cellato_batch_st* cellato_batch_t;

typedef struct {
    int rule;                /* cellato_rule */
    int x_cells, y_cells;    /* accepted by cellato_check_dims for the batch's layout */
    int steps;               /* this grid's steps per launch of the batch (>= 0) */
    void* planes_a[8];       /* input planes (first rule_planes entries used) */
    void* planes_b[8];       /* second buffer of the ping-pong */
} cellato_batch_grid;

/* Plans a batch: grids of one rule advance k_per_rule[rule] steps per round
 * (k_per_rule has n_k_per_rule entries; NULL, 0 or missing entries: 8).  All
 * rounds of all grids of one rule are ONE persistent kernel launch, in which a
 * grid's next round starts as soon as its previous round is done; the rules'
 * launches are parallel branches of one CUDA graph (built and instantiated
 * here).  Allocates the work lists on the device.  Grids' steps count from 0
 * (step parity as a run with t0 = 0).  A bounded device wait of the persistent
 * kernel that gives up is counted by cellato_device_wait_timeouts. */
int cellato_batch_create(int layout, int word_bits, const cellato_batch_grid* grids, int n_grids,
                         const int* k_per_rule, int n_k_per_rule, cellato_batch_t* out);
/* One graph launch: every grid advances its `steps` (ping-pong a -> b -> ...). */
int cellato_batch_launch(cellato_batch_t batch, cellato_stream_t stream);
/* 1 when grid's result is in planes_b after a launch (odd number of rounds). */
int cellato_batch_result_in_b(cellato_batch_t batch, int grid, int* in_b);
/* Kernel launches in the graph and work items (tiles x rounds) of the batch. */
int cellato_batch_info(cellato_batch_t batch, int* kernel_launches, long long* work_items);
int cellato_batch_destroy(cellato_batch_t batch);

/* ---- batched run without device allocation ------------------------------
 * No counterpart in the reference.  For callers that must not allocate device
 * memory -- a host framework or plugin host that owns all device memory through
 * its own pool, a latency-critical loop that cannot afford cudaMalloc's implicit
 * synchronisation, code held to a fixed device-memory budget.  Runs the same
 * batched temporal kernels as cellato_batch_create + cellato_batch_launch (same
 * results), with the work list kept in a fixed array in the library's device
 * memory (CELLATO_NOALLOC_MAX_GRIDS descriptors and CELLATO_NOALLOC_MAX_ITEMS
 * work items, about 1.2 MB, held by every GPU that loads the library until the
 * process exits) instead of a cudaMalloc'd one; no CUDA graph, stream or event
 * is created, the rules' persistent kernels are launched in order on `stream`.
 * Calls no cudaMalloc or cudaFree.
 *   - The work list is copied from host memory the library does not pin, so
 *     the call waits for the work already queued on `stream`; a stream being
 *     captured into a CUDA graph is refused with CELLATO_EINVAL.
 *   - grids: as for cellato_batch_create; result_in_b: n_grids ints (host),
 *     set to 1 where a grid's result is in planes_b.
 *   - More than CELLATO_NOALLOC_MAX_GRIDS grids or CELLATO_NOALLOC_MAX_ITEMS
 *     work items (tiles x rounds over the batch): CELLATO_EINVAL, nothing runs.
 *   - The first call on a device looks up the array's device address (with
 *     cudaGetSymbolAddress) and caches it for the process; do not use this
 *     entry point on a device after cudaDeviceReset.
 *   - All calls share the array and it keeps the last call's work list; each
 *     call writes the whole list it uses and clears the counters its kernels
 *     count from zero, before its kernels (stream-ordered).
 *     Calls whose work can overlap on the GPU (other streams, other threads)
 *     race on the array: serialise them. */
#define CELLATO_NOALLOC_MAX_GRIDS 1024
#define CELLATO_NOALLOC_MAX_ITEMS 65536
int cellato_batch_run_noalloc(int layout, int word_bits, const cellato_batch_grid* grids, int n_grids,
                              const int* k_per_rule, int n_k_per_rule, cellato_stream_t stream, int* result_in_b);

/* Largest tile_rows the temporal kernel accepts for (rule, layout, word_bits)
 * at the given words_per_lane (as cellato_tune) on the current device, or a
 * negative status. */
int cellato_temporal_max_tile_rows(int rule, int layout, int word_bits, int words_per_lane);

/* ---- whole-grid operations ----------------------------------------------- */

/* The reference's grid checksum computed from the planes on the device
 * (replaces standard_grid::get_checksum, include/memory/standard_grid.hpp:179-212,
 * which needs the grid converted to one state value per cell on the host):
 * sums[ty*4 + tx] = sum of the state values (not indices) of the cells of tile
 * (tx, ty) of the 4 x 4 partition into ceil(X/4) x ceil(Y/4) tiles.  The
 * reference prints the 16 sums joined by '-'.  sums: 16 uint64 in DEVICE
 * memory, overwritten (stream-ordered, no allocation). */
int cellato_checksum(int rule, int layout, int word_bits, const void* const* planes, int x_cells, int y_cells,
                     unsigned long long* sums, cellato_stream_t stream);

/* Full-grid diff: the number of cells whose state differs between two grids
 * of nb planes of plane_bytes each, in the same layout and word size (a cell
 * is the same bit position in every plane of either grid).  *count: one uint64
 * in DEVICE memory, overwritten (stream-ordered, no allocation).  Replaces
 * comparing two grids cell by cell after to_standard on the host (as the
 * reference's tests do, include/tests/bit_planes_grid.hpp:135-476). */
int cellato_diff_cells(int nb, const void* const* planes_a, const void* const* planes_b, size_t plane_bytes,
                       unsigned long long* count, cellato_stream_t stream);

/* ---- the bit_array layout --------------------------------------------------
 * The reference's third layout (include/memory/bit_array_grid.hpp:80-322): a
 * cell's nb index bits side by side, cells in row-major order, cpw =
 * array_word_bits / nb cells per word, cell i in word i / cpw at bit
 * (i % cpw) * nb; x_cells must be a multiple of cpw.  This library runs the
 * steps on bit planes: a bit_array grid is converted on the device when a run
 * starts and back when it ends (the C++ bit_array traverser does this), with
 * the results of the reference's bit_array evaluator
 * (include/evaluators/bit_array.hpp:73-105).  The planes' own layout and word
 * size must be accepted by cellato_check_dims as well. */

/* Bytes of the bit_array words of an X x Y grid, or 0 for bad arguments. */
size_t cellato_bit_array_bytes(int nb, int array_word_bits, int x_cells, int y_cells);
/* bit_array words (device) -> nb device planes in (layout, word_bits).
 * Stream-ordered, no allocation. */
int cellato_bit_array_to_planes(int nb, int array_word_bits, const void* array, int x_cells, int y_cells, int layout,
                                int word_bits, void* const* planes, cellato_stream_t stream);
/* nb device planes -> bit_array words (device).  Stream-ordered, no allocation. */
int cellato_planes_to_bit_array(int nb, int layout, int word_bits, const void* const* planes, int x_cells,
                                int y_cells, int array_word_bits, void* array, cellato_stream_t stream);

/* State value of dictionary index `index` of a rule (index_to_state,
 * include/memory/state_dictionary.hpp:10-70). */
int cellato_rule_state_value(int rule, int index, long long* value);

/* Seeded random initial state written straight into nb device planes.  Cell
 * (x, y) gets index #{i : thresholds[i] <= u}, u = upper 32 bits of the
 * SplitMix64 output at seed + (y*X + x + 1) * 0x9E3779B97F4A7C15 (ascending
 * thresholds, at most 31, fewer than 2^nb).  thresholds[i] =
 * floor(P(index <= i) * 2^32) gives the indices their probabilities.  This is
 * the library's own generator, not the reference's std::mt19937
 * (include/memory/grid_utils.hpp:36-60); stream-ordered, no allocation. */
int cellato_fill_random(int layout, int word_bits, int nb, void* const* planes, int x_cells, int y_cells,
                        unsigned long long seed, const uint32_t* thresholds, int n_thresholds,
                        cellato_stream_t stream);

/* ---- simulation server: continuous batching of many requests ------------
 * No counterpart in the reference (one grid per CLI run).  A request is one
 * grid of one automaton advanced `steps` steps from step 0; the server keeps
 * its planes resident on the device from admission to completion.
 *   - Admission: strict FIFO in submission order while the planes of the
 *     resident requests fit in hbm_cap_bytes (a stream-ordered memory pool owned
 *     by the server holds them).
 *   - Iteration (cellato_server_iterate): the resident requests, oldest first,
 *     are activated while their temporal tiles fit in tile_budget; each active
 *     request advances up to chunk_rounds rounds of k steps.  The rounds of
 *     one automaton are one persistent batched launch over the tiles of every
 *     active request of it (a request's next round starts when its previous
 *     round is done), the automata on parallel streams.  Requests join and
 *     leave between iterations, at any step count.
 *   - Completion: a finished request's checksum (as cellato_checksum) is
 *     computed on the device and copied back; cellato_server_poll returns it.
 *     Without `keep` its planes are freed at once; with `keep` they stay,
 *     readable through cellato_server_planes, until cellato_server_release.
 * Results are identical to cellato_run_temporal on each grid alone with the
 * same k.  A server is used from one host thread at a time; all its device work
 * is ordered on its own streams on the device current at creation. */

typedef struct cellato_server_st* cellato_server_t;

typedef struct {
    int layout;                       /* cellato_layout */
    int word_bits;                    /* 32 or 64 */
    unsigned long long hbm_cap_bytes; /* resident plane bytes; 0: 80% of the device's memory */
    int tile_budget;                  /* temporal tiles per round over all active requests; 0: 32 per SM */
    int chunk_rounds;                 /* rounds per request per iteration; 0: 4 */
    int max_inflight;                 /* iterations queued on the device at once; 0: 2 */
    const int* k_per_rule;            /* temporal depth per rule id, 1..32 (copied at creation);
                                         NULL, 0 or ids past n_k_per_rule: 16 */
    int n_k_per_rule;
} cellato_server_config;

typedef struct {
    long long id;
    int rule;
    int x_cells, y_cells, steps;
    int result_in_b;                  /* buffer holding the result (requests with keep) */
    unsigned long long checksum[16];
    double submit_s;                  /* server clock (seconds since creation) at submission */
    double done_s;                    /* server clock when the host saw the result */
} cellato_server_result;

typedef struct {
    long long waiting;                /* submitted, not admitted */
    long long running;                /* admitted, steps left */
    long long active;                 /* advanced by the last iteration */
    long long completed_unpolled;
    unsigned long long resident_bytes, hbm_cap_bytes;
    long long iterations, kernel_launches;
    double cell_steps;                /* cell updates enqueued since creation */
    long long pool_trims;             /* times a plane allocation found the pool fragmented: issued frees
                                         were completed, unused blocks returned, the allocation retried */
    long long memory_waits;           /* times admitted requests found no device memory even then: they
                                         went back to the head of the queue and the cap fell to the bytes
                                         resident (hbm_cap_bytes shows the current cap) */
} cellato_server_stats;

int cellato_server_create(const cellato_server_config* config, cellato_server_t* out);
/* Submit a request whose initial state is cellato_fill_random(seed, thresholds)
 * (thresholds as there; NULL with n_thresholds = 0: all cells index 0). */
int cellato_server_submit_random(cellato_server_t server, int rule, int x_cells, int y_cells, int steps,
                                 unsigned long long seed, const uint32_t* thresholds, int n_thresholds, int keep,
                                 long long* id);
/* Submit a request whose initial state is given as rule_planes host planes in
 * the server's layout (copied at submission). */
int cellato_server_submit_planes(cellato_server_t server, int rule, int x_cells, int y_cells, int steps,
                                 const void* const* host_planes, int keep, long long* id);
/* Submit a request resumed from a snapshot: host planes of the state reached
 * at step number t0 (cellato_server_snapshot's next_step), `steps` steps
 * still to run.  The step parity continues from t0 as if never interrupted. */
int cellato_server_submit_resume(cellato_server_t server, int rule, int x_cells, int y_cells, int steps, int t0,
                                 const void* const* host_planes, int keep, long long* id);
/* Snapshot (checkpoint) of a request on the device: waits for the server's
 * queued iterations, copies the planes of the request's current state into
 * rule_planes host buffers of x*y/8 bytes, and sets *steps_done (steps applied
 * since submission) and *next_step (t0 + steps_done).  The request keeps
 * running.  A request not yet admitted has no device state: CELLATO_EINVAL. */
int cellato_server_snapshot(cellato_server_t server, long long id, void* const* host_planes, int* steps_done,
                            int* next_step);
/* Removes a request at any stage (waiting, running, or completed with keep)
 * and frees its planes, after the server's queued work; a result of it that
 * cellato_server_poll has not returned yet is dropped.  Snapshot, cancel and
 * resume later is preemption without recomputation. */
int cellato_server_cancel(cellato_server_t server, long long id);
/* One scheduling iteration: collect finished work, admit, plan and enqueue one
 * chunk for the active requests.  Blocks only while max_inflight iterations are
 * queued (or, with nothing to run, until the oldest queued one completes).
 * *active = requests advanced by this iteration. */
int cellato_server_iterate(cellato_server_t server, int* active);
/* Moves up to `max` completed requests into out[]; *n = how many. */
int cellato_server_poll(cellato_server_t server, cellato_server_result* out, int max, int* n);
/* Device planes of a completed request submitted with keep (rule_planes entries). */
int cellato_server_planes(cellato_server_t server, long long id, void** planes);
/* Frees a completed request's planes (requests with keep). */
int cellato_server_release(cellato_server_t server, long long id);
int cellato_server_stats_get(cellato_server_t server, cellato_server_stats* stats);
/* Waits for all queued work and frees everything the server holds. */
int cellato_server_destroy(cellato_server_t server);

#ifdef __cplusplus
}
#endif

#endif /* CELLATO_B200_H */
