/*
 * vfb_oracle.h -- CPU restatement of VFB's cached bottom-up LTL enumeration.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product (the vfb_b200 package, its
 * CUDA library or CLI) links, loads or calls this code.  It is the checker for
 * the GPU path (tests, the smoke check) and the timed CPU baseline of bench.py.
 *
 * What it restates (reference file:line):
 *   operator semantics on characteristic sets  LTL_BS.cu:183-238, ltl_nocache.cu:95-150
 *   126-bit uniqueness key (exact / relaxed 1,2,3) LTL_BS.cu:30-110
 *   two-level hash-set dedup = exact membership on the normalised (h,l) pair
 *                                               LTL_BS.cu:251-269, hash_set.cuh:193-254
 *   solution test                               LTL_BS.cu:316-319
 *   level / operator / size-split structure     LTL_BS.cu:1226-1488
 *   formula numbering (canonical order)         ltl_nocache.cu:169-224, 248-287
 *   RPN evaluation                              ltl_nocache.cu:78-161
 */
#ifndef VFB_ORACLE_H
#define VFB_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_MAX_TRACES 128
#define ORC_MAX_VARS 64
#define ORC_MAX_SIZE 32

/* enumeration order */
#define ORC_MODE_CANONICAL 0  /* nocache numbering order, all U splits */
#define ORC_MODE_REFCOMPAT 1  /* LTL_BS launch structure incl. even-pair U subset */

/* status */
#define ORC_FOUND 0
#define ORC_NOT_FOUND 1
#define ORC_LIMIT 2
#define ORC_BAD_INPUT 3

typedef struct {
    int num_traces;            /* positives first, then negatives */
    int num_pos;
    int num_vars;
    int max_size;              /* 1..32 */
    int rlx_type;              /* 1, 2 or 3: used only when sum of lengths > 126 */
    int mode;                  /* ORC_MODE_* */
    int threads;               /* 1 = scalar oracle; >1 = OpenMP port */
    int64_t ref_max_pitch;     /* cudaDevAttrMaxPitch assumed by ref-compat chunking */
    uint64_t max_rows;         /* row budget; exceeding it returns ORC_LIMIT */
    const uint8_t *len;        /* [num_traces], 1..64 */
    const uint64_t *atoms;     /* [num_vars][num_traces] proposition words */
    int64_t *trace;            /* ref-compat launch log, 5 words per launch: cost, op
                                  (0..6, 7 = atoms), AllLTLs, StoredLTLs, ToBeChecked as
                                  printed before each launch (LTL_BS.cu:1193, 1230, ...) */
    int trace_cap;             /* launches the trace buffer can hold */
    int cost[8];               /* operator costs c1..c8 of LTL_BS (p ~ & | X F G U); 0 = 1.
                                  Levels are then costs: max_size is the maximum cost */
    int neg_type;              /* 1: ~ of any formula; 2: ~ of propositions only; 0 = 1 */
} orc_problem;

typedef struct {
    int status;
    int size;                  /* formula size if found, else last level reached */
    int rpn_len;
    int16_t rpn[ORC_MAX_SIZE]; /* >= 0: proposition; < 0: -(1 + op index in "~&|XFGU") */
    uint64_t level_rows[ORC_MAX_SIZE + 1];   /* unique rows per level (final level: up to the solution) */
    uint64_t level_cands[ORC_MAX_SIZE + 1];  /* candidates evaluated per level */
    uint64_t solution_index;   /* canonical candidate index of the solution within its level */
    uint64_t total_rows;
    double seconds;
    int trace_len;             /* launches written to problem->trace */
} orc_result;

/* Solve one instance.  Returns result->status. */
int orc_solve(const orc_problem *p, orc_result *r);

/* Solve, then, when nothing is found up to max_size, the BS stage of
 * LTL_BS.cu:870-1067 up to size bs_max: ~ & | combinations of the cached
 * formulas over their step-0 vectors (deterministic restatement, see the
 * source).  Sizes above max_size report BS entries in level_rows and
 * candidates in level_cands.  Needs at most 64 traces (ORC_LIMIT otherwise). */
int orc_solve_bs(const orc_problem *p, int bs_max, orc_result *r);

/* Exhaustive search in ltl_nocache numbering order (no cache, no dedup).
 * Returns the first formula (lowest number) that is a solution, or
 * ORC_NOT_FOUND / ORC_LIMIT when max_formulas candidates were evaluated. */
int orc_exhaustive(const orc_problem *p, uint64_t max_formulas, orc_result *r);

/* Evaluate an RPN token string on every trace; writes one word per trace into
 * cs_out (may be NULL).  Returns 1 if it is a solution, 0 if not, -1 if the RPN
 * is malformed. */
int orc_eval_rpn(const orc_problem *p, const int16_t *rpn, int rpn_len, uint64_t *cs_out);

/* The 126-bit key of one characteristic set (LTL_BS.cu:30-110), normalised the
 * way the reference's two-level hash set identifies keys. */
void orc_make_key(const orc_problem *p, const uint64_t *cs, uint64_t *h, uint64_t *l);

/* Apply one operator to characteristic sets (op index into "~&|XFGU"). */
void orc_apply(const orc_problem *p, int op, const uint64_t *l, const uint64_t *r, uint64_t *out);

/* Reference temp-buffer capacity (rows) used by ref-compat chunking. */
int64_t orc_ref_temp_capacity(const orc_problem *p);

#ifdef __cplusplus
}
#endif
#endif
