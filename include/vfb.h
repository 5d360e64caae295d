/*
 * vfb.h -- C ABI of the B200-native VFB engine (libvfb_b200.so).
 *
 * Learns the smallest LTL formula over  AP | ~f | f&g | f|g | Xf | Ff | Gf | fUg
 * that holds at step 0 of every positive trace and fails at step 0 of every
 * negative trace, by bottom-up enumeration with a per-level characteristic-set
 * cache and semantic deduplication on one GPU.
 *
 * Plain C types only; no exceptions or C++ types cross this boundary.  Every
 * entry point returns a vfb_status.  A context is not thread-safe: use one per
 * host thread (or serialise calls).
 *
 * Reference interfaces these entry points replace (SynthesisLab/VFB):
 *   vfb_solve        std::string LTL(maxLen, inputData, traceLen, traceLength)
 *                    ltl_nocache.cu:319-446, with the search of
 *                    std::string LTLI(...) LTL_BS.cu:1069-1532 (cached,
 *                    deduplicated enumeration); same input layout
 *                    inputData[trace*numVar + var] (ltl_nocache.cu:51-65)
 *   vfb_read_json    readJsonFile  ltl_nocache.cu:35-76
 *   vfb_format_infix LTLToString   ltl_nocache.cu:289-317
 *   vfb_batch_solve  no counterpart (the reference solves one instance per
 *                    process); results equal one vfb_solve per instance
 *   vfb_create / vfb_destroy  replace the reference's process-global state
 *                    (__constant__ symbols, cudaMalloc'd caches) with a context
 */
#ifndef VFB_H
#define VFB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define VFB_MAX_SIZE 32      /* formula size limit (ltl_nocache.cu:11) */
#define VFB_MAX_TRACES 128
#define VFB_MAX_VARS 64
#define VFB_MAX_LENGTH 64    /* one uint64 word per trace (ltl_nocache.cu:12) */

typedef enum {
  VFB_OK = 0,            /* formula found */
  VFB_NOT_FOUND = 1,     /* no formula up to max_size ("Not found !", ltl_nocache.cu:439) */
  VFB_LIMIT = 2,         /* input outside the supported limits */
  VFB_OOM = 3,           /* device memory budget exhausted */
  VFB_DEVICE_ERROR = 4,  /* CUDA error, missing device or kernel image */
  VFB_TIMEOUT = 5,       /* reserved for the serving loop */
  VFB_BAD_INPUT = 6      /* malformed arguments or JSON */
} vfb_status;

/* Operator tokens in results: token >= 0 is a proposition index; token < 0 is
 * -(1 + i) for operator i of "~&|XFGU" (the reference's Op order, LTL_BS.cu:17). */
#define VFB_TOK_OP(i) (-(1 + (i)))

typedef struct {
  int device;              /* CUDA device ordinal */
  size_t mem_limit_bytes;  /* device memory budget of one solve/batch (0: 90% of the memory
                              free at creation, counting what the process's stream-ordered
                              pool holds unused) */
  int verbose;             /* 1: per-level progress lines on stderr */
  int profile;             /* 1: time every kernel of the level step with CUDA events
                              (see vfb_profile_read); adds one event pair per kernel */
} vfb_opts;

/* One learning problem.  Layout as ltl_nocache's readJsonFile: words[i*num_vars + v]
 * holds proposition v on trace i (bit t = value at step t); traces 0..num_pos-1
 * are positive, the rest negative; lengths[i] is trace i's length (1..64). */
typedef struct {
  int num_vars;
  int num_traces;
  int num_pos;
  const uint64_t *words;
  const int *lengths;
  int max_size;            /* 1..32 */
  int rlx_type;            /* relaxed-uniqueness rule when total trace bits exceed 126:
                              1 strided sample, 2 proportional prefix, 3 hash (default,
                              0 means 3); LTL_BS.cu:30-110 */
} vfb_instance;

typedef struct {
  vfb_status status;
  int size;                          /* formula size, or last level searched */
  int rpn_len;
  int16_t rpn[VFB_MAX_SIZE];         /* RPN tokens, see VFB_TOK_OP */
  uint64_t level_rows[VFB_MAX_SIZE + 1];   /* unique characteristic sets per size (index = size);
                                              the final size counts up to the solution */
  uint64_t level_cands[VFB_MAX_SIZE + 1];  /* candidates evaluated per size */
  uint64_t total_rows;               /* sum of level_rows */
  uint64_t solution_index;           /* canonical index of the solution within its size */
  double seconds;                    /* wall time of the call (batch: of the whole batch) */
  double device_seconds;             /* device timeline from the first upload to the last
                                        result read (CUDA events on the engine's stream) */
  uint64_t h2d_bytes, d2h_bytes;     /* bytes copied host->device / device->host by the call */
  uint64_t kernel_launches;          /* kernels this call launched */
} vfb_result;

vfb_status vfb_create(void **ctx, const vfb_opts *opts);
void vfb_destroy(void *ctx);

/* The cached search (LTLI LTL_BS.cu:1069-1532 in the canonical order of
 * ltl_nocache).  Buffers grow up to opts->mem_limit_bytes; when a level's
 * rows cannot be held, that level's candidates are still tested as solutions
 * without being stored (the reference's onTheFly mode, LTL_BS.cu:331-349):
 * a solution found there is returned as usual with level_rows[size] = 0,
 * otherwise the call ends with VFB_LIMIT and the sizes it stored. */
vfb_status vfb_solve(void *ctx, const vfb_instance *inst, vfb_result *out);

/* Solves n independent instances together; out[i] equals vfb_solve(inst[i])
 * under the same memory budget.  When the budget cannot hold every instance
 * at once, instances wait for memory the others free, and an instance that
 * cannot get its buffers while the others hold theirs is solved alone after
 * them. */
vfb_status vfb_batch_solve(void *ctx, const vfb_instance *inst, int n, vfb_result *out);

/* vfb_solve with the operator costs of LTL_BS (LTLI LTL_BS.cu:1069-1532,
 * arguments c1..c8 and NegType of its main, 1612-1666): costs[0..7] = cost of
 * a proposition, ~, &, |, X, F, G, U (each >= 1); the levels are then costs:
 * a formula's cost is the sum of its symbols' costs, inst->max_size is the
 * largest cost searched, and size / level_rows / level_cands are indexed by
 * cost (levels below costs[0] are empty).  neg_type 1 lets ~ apply to any
 * formula, 2 to propositions only.  The order within a cost is the reference's
 * launch order: ~ & | X F G U, & and | over cost splits (i, k - c - i) with
 * i <= k - c - i, U over every split, left index major.  Unit costs and
 * neg_type 1 are exactly vfb_solve. */
vfb_status vfb_solve_costs(void *ctx, const vfb_instance *inst, const int *costs, int neg_type,
                           vfb_result *out);

/* vfb_solve, then, when nothing is found up to inst->max_size, the BS stage
 * of LTL_BS (BS LTL_BS.cu:870-1067) up to size bs_max_size: ~ & |
 * combinations of the cached formulas over their step-0 vectors (bit i = the
 * formula holds at step 0 of trace i), searched in canonical order (sizes
 * ascending; ~ over size c-1, then & and | over size splits i <= (c-1)/2,
 * left index major) with the first occurrence of each vector kept; the first
 * combination whose vector is exactly the positive traces' is returned.
 * Sizes above max_size report vector entries in level_rows and combinations
 * in level_cands.  At most 64 traces (VFB_LIMIT otherwise). */
vfb_status vfb_solve_bs(void *ctx, const vfb_instance *inst, int bs_max_size, vfb_result *out);

/* Cache-free search, replacing string LTL(...) of ltl_nocache.cu:319-446:
 * every formula of each size is evaluated in the numbering order of
 * numberToFormula (ltl_nocache.cu:169-224) with no cache and no
 * deduplication, and the first solution of that order is returned (the
 * reference returns a solution of the same size and root operator block;
 * which one within the block is a race there).  level_cands[k] counts the
 * formulas evaluated of size k; level_rows stays 0.  Sizes whose formula
 * count exceeds 2^62 are not searched (VFB_LIMIT). */
vfb_status vfb_solve_exhaustive(void *ctx, const vfb_instance *inst, vfb_result *out);

/* Solve without allocating.  No counterpart in the reference.
 *
 * For callers that may not allocate device (or pinned host) memory while they
 * run -- a process whose device heap is owned by another allocator, a
 * latency-critical loop that cannot take cudaMalloc's implicit
 * synchronisation, a driver heap closed after start-up.  Needs no context:
 * it runs the same kernels as vfb_solve on the current device and the legacy
 * default stream, with every device buffer carved from one static array of
 * VFB_NOALLOC_SCRATCH_BYTES that the library's module holds on every GPU that
 * loads it, until the process exits.  Buffers do not grow: the array holds a
 * hash set of 2^19 slots, a bitmap of 2^25 candidates per size, 2^19
 * owner-list entries and about 40 MiB of level cache, which holds
 * 40 MiB / (8*TP + 8) characteristic sets (TP = traces rounded up to even:
 * about 127,000 at 40 traces, 40,000 at 128); at most about 2^18 distinct
 * sets in all (the hash set is planned at most half full); a search that needs
 * more stops with VFB_OOM and a message on stderr.  The first call on a device
 * resolves the array's address and should come before any stream capture;
 * after a device reset the next call resolves it again.  All calls share the
 * array (each one clears what must start empty); calls that overlap on the
 * GPU race, so serialise them.  Results equal vfb_solve's for every instance
 * that fits; device_seconds is not measured (0). */
#define VFB_NOALLOC_SCRATCH_BYTES (64u << 20)
vfb_status vfb_solve_noalloc(const vfb_instance *inst, vfb_result *out);

/* ------------------------------------------------------------ serving loop
 * Continuous batching (no counterpart in the reference, which solves one
 * instance per process).  vfb_serve_open keeps `slots` instances resident on
 * the device (traces up to max_traces).  vfb_serve_submit queues a request
 * (the instance is copied).  Each vfb_serve_step admits queued requests into
 * free slots while the bytes the resident instances are projected to hold
 * after their next level (last level-over-level growth) stay under
 * budget_frac of the memory budget (the head of the queue is admitted
 * whenever no slot is busy; past that, a light request is still admitted
 * when its first buffers fit the budget beside what is live), builds one
 * more level of every resident instance, and returns the finished ones (up
 * to cap) with their tags; results equal vfb_solve's.  A growth that finds
 * the memory held by other requests waits for it; requests that can only
 * wait for one another (none can go on, or two or more have waited 32
 * steps) give way: the least advanced one is evicted and queued again at
 * the front, to start over.  An instance whose buffers would grow past
 * request_bytes finishes with VFB_LIMIT and the sizes it completed.
 * *active / *queued (may be NULL) report the slots in use and the requests
 * waiting.  A request that cannot be admitted finishes with its status.
 * A level of more than step_candidates candidates is built over several
 * steps (slices of its operator tiles), so one large request does not hold
 * the others' steps for long.  vfb_serve_limits sets budget_frac (default
 * 0.8), request_bytes (0, the default: a quarter of the budget) and
 * step_candidates (default 2^23; 0: whole levels) for the next
 * vfb_serve_open and the open session.  vfb_serve_open takes the memory
 * budget (less what the engine holds live) from the device in one
 * allocation, halved until it can be had, and the session's buffers are
 * carved out of it, so that growth inside a step maps no new device memory;
 * vfb_serve_close gives it back to the engine's pool (vfb_destroy returns
 * the pool's memory to the device). */
typedef struct {
  uint64_t tag;
  vfb_result result;
} vfb_served;

vfb_status vfb_serve_open(void *ctx, int slots, int max_traces);
vfb_status vfb_serve_limits(void *ctx, double budget_frac, uint64_t request_bytes,
                            uint64_t step_candidates);
vfb_status vfb_serve_submit(void *ctx, const vfb_instance *inst, uint64_t tag);
vfb_status vfb_serve_step(void *ctx, vfb_served *done, int cap, int *ndone, int *active, int *queued);
void vfb_serve_close(void *ctx);

/* Per-kernel profile accumulated since vfb_create (profile=1 only).  name,
 * number of launches, total device milliseconds (CUDA events around each
 * launch) and the algorithmic bytes those launches had to move (operand rows
 * read once, one 32-byte slot sector per hash probe, rows and indices written,
 * bitmap words).  Returns the number of kernels written (at most cap). */
typedef struct {
  char name[32];
  uint64_t launches;
  double ms;
  double bytes;
} vfb_kernel_stat;

int vfb_profile_read(void *ctx, vfb_kernel_stat *out, int cap);
void vfb_profile_reset(void *ctx);

/* Launch shape of the candidate kernel (k_p1) per level band (no counterpart
 * in the reference, whose processOperator launches use fixed block sizes,
 * LTL_BS.cu:1284-1305).  Band b holds the levels of 4^b .. 4^(b+1)-1
 * candidates, the last band every larger level.  A tile is 128 rows of one
 * operand level against `rows` staged rows of the other; small levels are cut
 * into shorter tiles until they have 2^tiles_log2 of them; `blocks` CTAs take
 * the tiles.  Zero in a field selects the built-in choice (rows 16,
 * tiles_log2 12, every resident CTA).  Results never depend on the shape. */
#define VFB_TUNE_BANDS 16
typedef struct {
  uint8_t rows[VFB_TUNE_BANDS];         /* staged rows per tile: 1, 2, 4, .. 32 (above 16 acts as 16) */
  uint8_t tiles_log2[VFB_TUNE_BANDS];   /* tile count to reach by shorter tiles, log2 (1..40) */
  uint16_t blocks[VFB_TUNE_BANDS];      /* CTAs of the level's launch */
  float ms[VFB_TUNE_BANDS];             /* vfb_autotune: k_p1 time of the chosen shape summed
                                           over the sample's levels in the band (0: none) */
  float ms_default[VFB_TUNE_BANDS];     /* vfb_autotune: the same with the built-in shape */
  uint32_t levels[VFB_TUNE_BANDS];      /* vfb_autotune: the sample's levels in the band */
} vfb_tune;

/* The shape every later solve, batch and served request of ctx uses
 * (NULL: the built-in shape everywhere). */
vfb_status vfb_tune_set(void *ctx, const vfb_tune *tune);
vfb_status vfb_tune_get(void *ctx, vfb_tune *tune);

/* Autotuner: solves the n sample instances once per candidate shape (staged
 * rows 2/4/8/16 x tile targets 2^8/2^10/2^12/2^14 x every resident CTA or one
 * per SM), `reps` times each (>= 1), timing k_p1 at every level with CUDA events;
 * each band takes the shape with the least time over the sample's levels in
 * that band (bands without a level keep the built-in shape).  The result is
 * installed in ctx (as vfb_tune_set) and written to *out when out is not
 * NULL.  Every sample solve must return the same result under every shape,
 * else VFB_DEVICE_ERROR. */
vfb_status vfb_autotune(void *ctx, const vfb_instance *sample, int n, int reps, vfb_tune *out);

/* Seeded synthetic instance (no counterpart in the reference, which ships no
 * benchmark inputs): rejection-samples n_pos + n_neg traces with lengths
 * uniform in [len_lo, len_hi] and i.i.d. Bernoulli(p) bits, labelled by a
 * formula of planted_size drawn uniformly with the ltl_nocache numbering
 * (ltl_nocache.cu:169-224, 248-287).  rng_state is a xoshiro256** state (4
 * words) advanced in place.  Outputs words[i*num_vars+v], lengths[i] (positives
 * first) and the planted formula's RPN tokens.  Returns 0, or -1 on bad sizes. */
int vfb_synth_planted(uint64_t *rng_state, int num_vars, int planted_size, int n_pos, int n_neg,
                      int len_lo, int len_hi, double p, int max_draws_per_trace, uint64_t *words_out,
                      int *lengths_out, int16_t *rpn_out, int *rpn_len);

/* Human-readable name of a status. */
const char *vfb_status_str(vfb_status s);

/* ----------------------------------------------------------- trace JSON input
 * Parses a trace file in the reference's JSON schema (keys
 * number_atomic_propositions, number_traces, number_positive_traces,
 * max_length_traces, atomic_propositions, positive_traces, negative_traces).
 * On success *out is a library-owned problem; free it with vfb_json_free. */
typedef struct {
  vfb_instance inst;
  int max_length_traces;   /* the file's declared maximum length */
  char **names;            /* num_vars proposition names */
} vfb_json_problem;

vfb_status vfb_read_json(const char *path, vfb_json_problem **out, char *err, size_t errlen);
void vfb_json_free(vfb_json_problem *p);

/* Infix text of a result's formula in the reference's notation: "~(x)",
 * "X(x)", "(l) & (r)", "(l) U (r)" (ltl_nocache.cu:289-317).  Writes at most
 * buflen bytes including the terminator; returns the full length needed, or
 * -1 if the RPN is malformed. */
int vfb_format_infix(const vfb_result *r, const char *const *names, char *buf, size_t buflen);

#ifdef __cplusplus
}
#endif
#endif
