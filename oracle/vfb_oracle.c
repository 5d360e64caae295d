/*
 * vfb_oracle.c -- CPU restatement of VFB's cached bottom-up LTL enumeration.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the GPU path and the timed CPU
 * baseline.  The product never links or loads it.  See vfb_oracle.h for the
 * list of reference functions restated here.
 *
 * Enumeration order.  The reference resolves the dedup representative and the
 * reported solution with racy atomicCAS (LTL_BS.cu:319, hash_set.cuh:232), so
 * a deterministic order has to be fixed: the canonical order is the numbering
 * of ltl_nocache.cu (numberToFormula 169-224): levels by size; inside a level
 * the operator blocks ~ & | X F G U; binary blocks split by left size
 * ascending (& and | only up to floor((k-1)/2), U over every split 1..k-2);
 * left operand index major, right operand index minor.  The first candidate in
 * this order that yields a key represents it, and the first representative
 * that is a solution is returned.  ORC_MODE_REFCOMPAT instead walks the
 * candidate sequence of LTL_BS's launches (temp-buffer chunking
 * LTL_BS.cu:1248-1268, U evaluated as lUr/rUl for even pair indices only,
 * LTL_BS.cu:397-442 and 1454-1482); stale temp slots that the reference also
 * appends (LTL_BS.cu:1481) are not reproducible and are not modelled.
 */
#include "vfb_oracle.h"

#include <stdlib.h>
#include <string.h>
#include <time.h>
#ifdef _OPENMP
#include <omp.h>
#endif

enum { OP_NOT = 0, OP_AND, OP_OR, OP_X, OP_F, OP_G, OP_U, OP_NONE = 7 };
static const char OPCH[] = "~&|XFGU";

static inline int op_is_unary(int op) {
    return op == OP_NOT || op == OP_X || op == OP_F || op == OP_G;
}

static inline uint64_t len_mask(int L) {
    return L >= 64 ? ~0ULL : ((1ULL << L) - 1ULL);
}

static inline uint64_t suffix_or(uint64_t w) {
    w |= w >> 1;
    w |= w >> 2;
    w |= w >> 4;
    w |= w >> 8;
    w |= w >> 16;
    w |= w >> 32;
    return w;
}

/* "l U r" on one trace word: the doubling recurrence of LTL_BS.cu:222-233. */
static inline uint64_t until_word(uint64_t l, uint64_t r) {
    for (int s = 1; s <= 16; s <<= 1) {
        r |= l & (r >> s);
        l &= l >> s;
    }
    r |= l & (r >> 32);
    return r;
}

static inline uint64_t apply_word(int op, uint64_t l, uint64_t r, int L) {
    switch (op) {
    case OP_NOT: return ~l & len_mask(L);
    case OP_AND: return l & r;
    case OP_OR: return l | r;
    case OP_X: return l >> 1;
    case OP_F: return suffix_or(l);
    case OP_G: return l & ~suffix_or(~l & len_mask(L));
    default: return until_word(l, r);
    }
}

void orc_apply(const orc_problem *p, int op, const uint64_t *l, const uint64_t *r, uint64_t *out) {
    for (int i = 0; i < p->num_traces; ++i)
        out[i] = apply_word(op, l[i], r ? r[i] : 0, p->len[i]);
}

static int len_sum(const orc_problem *p) {
    int s = 0;
    for (int i = 0; i < p->num_traces; ++i) s += p->len[i];
    return s;
}

static inline uint64_t splitmix_fin(uint64_t x) {
    x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ULL;
    x = (x ^ (x >> 27)) * 0x94d049bb133111ebULL;
    return x ^ (x >> 31);
}

/* Place bit value v at position j of the 126-bit string (l: 0..62, h: 63..125). */
static inline int put_bit(uint64_t *h, uint64_t *l, int j, int v) {
    if (j < 63) { if (v) *l |= 1ULL << j; return 1; }
    if (j < 126) { if (v) *h |= 1ULL << (j - 63); return 1; }
    return 0;
}

static void make_key_s(const orc_problem *p, int S, const uint64_t *cs, uint64_t *ph, uint64_t *pl) {
    const int T = p->num_traces;
    uint64_t h = 0, l = 0;
    int j = 0;
    if (S > 126) {
        if (p->rlx_type == 1) {
            /* every stride-th step of every trace, trace-major (LTL_BS.cu:45-58) */
            const int stride = S / 126;
            for (int i = 0; i < T; ++i)
                for (int k = 0; k < p->len[i]; k += stride, ++j)
                    if (!put_bit(&h, &l, j, (int)((cs[i] >> k) & 1))) break;
        } else if (p->rlx_type == 2) {
            /* a length-proportional prefix of every trace (LTL_BS.cu:61-75) */
            for (int i = 0; i < T; ++i) {
                const int nb = (126 * p->len[i] + S) / S;
                for (int k = 0; k < nb; ++k, ++j)
                    if (!put_bit(&h, &l, j, k < 64 ? (int)((cs[i] >> k) & 1) : 0)) break;
            }
        } else {
            /* splitmix64 finaliser of each word, XOR-folded: first half of the
             * traces into h, the rest into l (LTL_BS.cu:78-87) */
            for (int i = 0; i < T; ++i) {
                const uint64_t x = splitmix_fin(cs[i]);
                if (i < T / 2) h ^= x; else l ^= x;
            }
        }
    } else {
        /* exact: all steps of all traces, trace-major (LTL_BS.cu:96-106) */
        for (int i = 0; i < T; ++i)
            for (int k = 0; k < p->len[i]; ++k, ++j)
                if (!put_bit(&h, &l, j, (int)((cs[i] >> k) & 1))) break;
    }
    /* The reference's set stores h and l in a WarpCore set whose empty/tombstone
     * keys (~0, ~0-1) are rejected with slot code 0 (hash_set.cuh:201-205), so
     * both invalid values identify the same pair component. */
    if (h == ~0ULL) h = ~0ULL - 1;
    if (l == ~0ULL) l = ~0ULL - 1;
    *ph = h;
    *pl = l;
}

void orc_make_key(const orc_problem *p, const uint64_t *cs, uint64_t *h, uint64_t *l) {
    make_key_s(p, len_sum(p), cs, h, l);
}

static int is_solution(const orc_problem *p, const uint64_t *cs) {
    for (int i = 0; i < p->num_pos; ++i)
        if (!(cs[i] & 1)) return 0;
    for (int i = p->num_pos; i < p->num_traces; ++i)
        if (cs[i] & 1) return 0;
    return 1;
}

/* ------------------------------------------------------------ key set (exact) */
typedef struct {
    uint64_t *h, *l;
    uint8_t *used;
    size_t cap, count;
} kset;

static inline size_t kslot(uint64_t h, uint64_t l, size_t mask) {
    uint64_t x = h * 0x9E3779B97F4A7C15ULL ^ (l + 0x632BE59BD9B4E019ULL);
    x ^= x >> 29;
    x *= 0xBF58476D1CE4E5B9ULL;
    x ^= x >> 32;
    return (size_t)x & mask;
}

static int kset_init(kset *s, size_t cap) {
    s->cap = cap;
    s->count = 0;
    s->h = (uint64_t *)malloc(cap * sizeof(uint64_t));
    s->l = (uint64_t *)malloc(cap * sizeof(uint64_t));
    s->used = (uint8_t *)calloc(cap, 1);
    return s->h && s->l && s->used;
}

static void kset_free(kset *s) {
    free(s->h);
    free(s->l);
    free(s->used);
    memset(s, 0, sizeof(*s));
}

static int kset_contains(const kset *s, uint64_t h, uint64_t l) {
    size_t m = s->cap - 1, i = kslot(h, l, m);
    while (s->used[i]) {
        if (s->h[i] == h && s->l[i] == l) return 1;
        i = (i + 1) & m;
    }
    return 0;
}

static int kset_grow(kset *s);

/* 1 if inserted, 0 if present, -1 on allocation failure */
static int kset_insert(kset *s, uint64_t h, uint64_t l) {
    if (2 * (s->count + 1) > s->cap && !kset_grow(s)) return -1;
    size_t m = s->cap - 1, i = kslot(h, l, m);
    while (s->used[i]) {
        if (s->h[i] == h && s->l[i] == l) return 0;
        i = (i + 1) & m;
    }
    s->used[i] = 1;
    s->h[i] = h;
    s->l[i] = l;
    s->count++;
    return 1;
}

static int kset_grow(kset *s) {
    kset n;
    if (!kset_init(&n, s->cap * 2)) { kset_free(&n); return 0; }
    for (size_t i = 0; i < s->cap; ++i)
        if (s->used[i]) kset_insert(&n, s->h[i], s->l[i]);
    kset_free(s);
    *s = n;
    return 1;
}

/* ------------------------------------------------------------------ row store */
typedef struct {
    uint64_t *cs;      /* n x T words */
    int8_t *op;
    int64_t *left, *right;
    uint64_t n, cap;
    int T;
} rows_t;

static int rows_reserve(rows_t *r, uint64_t want) {
    if (want <= r->cap) return 1;
    uint64_t nc = r->cap ? r->cap : 1024;
    while (nc < want) nc *= 2;
    uint64_t *cs = (uint64_t *)realloc(r->cs, nc * r->T * sizeof(uint64_t));
    if (!cs) return 0;
    r->cs = cs;
    int8_t *op = (int8_t *)realloc(r->op, nc);
    if (!op) return 0;
    r->op = op;
    int64_t *lf = (int64_t *)realloc(r->left, nc * sizeof(int64_t));
    if (!lf) return 0;
    r->left = lf;
    int64_t *rt = (int64_t *)realloc(r->right, nc * sizeof(int64_t));
    if (!rt) return 0;
    r->right = rt;
    r->cap = nc;
    return 1;
}

static void rows_free(rows_t *r) {
    free(r->cs);
    free(r->op);
    free(r->left);
    free(r->right);
    memset(r, 0, sizeof(*r));
}

/* ------------------------------------------------------------- search state */
typedef struct {
    const orc_problem *p;
    int T, S;
    rows_t rows;
    kset set;
    uint64_t lvl_start[ORC_MAX_SIZE + 2];
    uint64_t lvl_count[ORC_MAX_SIZE + 2];
    uint64_t cands;        /* candidates evaluated at the current level */
    int level;
    int found;
    int64_t found_row;
    uint64_t found_g;
    int error;             /* ORC_LIMIT on row budget / allocation failure */
    uint64_t *tmp;
    uint64_t all_ltls;     /* LTL_BS's AllLTLs counter (ref-compat trace) */
    int trace_len;
} search_t;

/* One LTL_BS progress line, printed before each launch. */
static void trace_launch(search_t *s, int cost, int op, uint64_t n_printed) {
    const orc_problem *p = s->p;
    if (p->trace && s->trace_len < p->trace_cap) {
        int64_t *e = p->trace + 5 * (size_t)s->trace_len;
        e[0] = cost;
        e[1] = op;
        e[2] = (int64_t)s->all_ltls;
        e[3] = (int64_t)s->rows.n;
        e[4] = (int64_t)n_printed;
        s->trace_len++;
    }
    s->all_ltls += n_printed;
}

static inline const uint64_t *row_cs(const search_t *s, int64_t r) {
    return s->rows.cs + (size_t)r * s->T;
}

/* Evaluate one candidate; returns 1 when the search must stop. */
static int process(search_t *s, int op, int64_t a, int64_t b) {
    const orc_problem *p = s->p;
    uint64_t *cs = s->tmp;
    const uint64_t g = s->cands++;
    orc_apply(p, op, row_cs(s, a), op_is_unary(op) ? NULL : row_cs(s, b), cs);
    uint64_t h, l;
    make_key_s(p, s->S, cs, &h, &l);
    int ins = kset_insert(&s->set, h, l);
    if (ins < 0) { s->error = ORC_LIMIT; return 1; }
    if (!ins) return 0;
    if (s->rows.n >= p->max_rows || !rows_reserve(&s->rows, s->rows.n + 1)) {
        s->error = ORC_LIMIT;
        return 1;
    }
    const uint64_t r = s->rows.n++;
    memcpy(s->rows.cs + r * s->T, cs, s->T * sizeof(uint64_t));
    s->rows.op[r] = (int8_t)op;
    s->rows.left[r] = a;
    s->rows.right[r] = b;
    s->lvl_count[s->level]++;
    if (is_solution(p, cs)) {
        s->found = 1;
        s->found_row = (int64_t)r;
        s->found_g = g;
        return 1;
    }
    return 0;
}

/* Operator cost (c2..c8 for ~ & | X F G U; c1 for a proposition). */
static inline int op_cost(const orc_problem *p, int op) {
    const int c = p->cost[1 + op];
    return c > 0 ? c : 1;
}
static inline int atom_cost(const orc_problem *p) { return p->cost[0] > 0 ? p->cost[0] : 1; }

/* ---------------------------------------------------------- level: canonical
 * Level k holds the formulas of cost k (with unit costs: of size k).  Blocks
 * ~ & | X F G U (LTL_BS.cu:1226-1488): a unary operator of cost c reads level
 * k - c; & and | of cost c read splits (i, k - c - i), i from the
 * propositions' cost while i <= k - c - i; U reads every split (i, k - c - i)
 * with both sides at least the propositions' cost; left index major.  ~ reads
 * only the propositions when neg_type is 2 (LTL_BS.cu:1237-1240). */
static int level_canonical(search_t *s, int k) {
    const orc_problem *p = s->p;
    const int c1 = atom_cost(p);
    for (int op = 0; op < 7; ++op) {
        const int w = op_cost(p, op);
        if (op_is_unary(op)) {
            const int L = k - w;
            if (L < c1) continue;
            if (op == OP_NOT && p->neg_type == 2 && L != c1) continue;
            const uint64_t u0 = s->lvl_start[L], un = s->lvl_count[L];
            for (uint64_t a = 0; a < un; ++a)
                if (process(s, op, (int64_t)(u0 + a), -1)) return 1;
            continue;
        }
        for (int i = c1; ; ++i) {
            const int j = k - w - i;
            if (j < c1 || (op != OP_U && i > j)) break;
            const uint64_t l0 = s->lvl_start[i], ln = s->lvl_count[i];
            const uint64_t r0 = s->lvl_start[j], rn = s->lvl_count[j];
            for (uint64_t a = 0; a < ln; ++a)
                for (uint64_t b = 0; b < rn; ++b)
                    if (process(s, op, (int64_t)(l0 + a), (int64_t)(r0 + b))) return 1;
        }
    }
    return 0;
}

/* Temp-buffer capacity of LTL_BS (rows): int(maxPitch/(8T) * 1.5) / 2 (LTL_BS.cu:1179-1183). */
int64_t orc_ref_temp_capacity(const orc_problem *p) {
    const int64_t pitch = p->ref_max_pitch > 0 ? p->ref_max_pitch : 2147483647LL;
    const int64_t cacheCap = (int64_t)((double)(pitch / (int64_t)(p->num_traces * 8)) * 1.5);
    return cacheCap / 2;
}

/* ------------------------------------------- level: LTL_BS launch structure */
static int level_refcompat(search_t *s, int k) {
    const int64_t temp = orc_ref_temp_capacity(s->p);
    const int64_t u0 = (int64_t)s->lvl_start[k - 1];
    const int64_t u1 = u0 + (int64_t)s->lvl_count[k - 1] - 1;
    for (int op = 0; op < 7; ++op) {
        if (op_is_unary(op)) {
            if (u1 < u0) continue;
            int64_t x = u0, y;
            do {
                y = x + ((temp - 1) < (u1 - x) ? (temp - 1) : (u1 - x));
                trace_launch(s, k, op, (uint64_t)(y - x + 1));
                for (int64_t a = x; a <= y; ++a)
                    if (process(s, op, a, -1)) return 1;
                x = y + 1;
            } while (y < u1);
            continue;
        }
        for (int i = 1; 2 * i <= k - 1; ++i) {
            const int j = k - 1 - i;
            const int64_t i1 = (int64_t)s->lvl_start[i], i2 = i1 + (int64_t)s->lvl_count[i] - 1;
            const int64_t i3 = (int64_t)s->lvl_start[j], i4 = i3 + (int64_t)s->lvl_count[j] - 1;
            const int64_t nl = i2 - i1 + 1;
            if (nl <= 0 || i4 < i3) continue;
            int64_t x = i3, y;
            do {
                const int64_t cw = (op == OP_U) ? temp / (2 * nl) - 1 : temp / nl - 1;
                y = x + (cw < (i4 - x) ? cw : (i4 - x));
                const int64_t w = y - x + 1;
                const int64_t n = w * nl;
                trace_launch(s, k, op, (uint64_t)(op == OP_U ? 2 * n : n));
                if (op != OP_U) {
                    for (int64_t t = 0; t < n; ++t)
                        if (process(s, op, i1 + t / w, x + t % w)) return 1;
                } else {
                    /* tid = 2*realTid < n: even pairs only, each as lUr then rUl */
                    for (int64_t t = 0; t < n; t += 2) {
                        const int64_t a = i1 + t / w, b = x + t % w;
                        if (process(s, OP_U, a, b)) return 1;
                        if (process(s, OP_U, b, a)) return 1;
                    }
                }
                x = y + 1;
            } while (y < i4);
        }
    }
    return 0;
}

/* ---------------------------------------------- level: canonical, OpenMP port */
typedef struct {
    uint64_t t;
    uint64_t h, l;
} pend_t;

/* Candidates of one (op, split) block, t-th in canonical order. */
typedef struct {
    int op;
    uint64_t l0, ln, r0, rn;
} block_t;

/* Blocks and batches of fewer chunks (of 4096 candidates) than this run on
 * the calling thread. */
#define ORC_PAR_MIN_CHUNKS 8

static int run_block_parallel(search_t *s, const block_t *bk) {
    const orc_problem *p = s->p;
    const int T = s->T;
    const uint64_t n = op_is_unary(bk->op) ? bk->ln : bk->ln * bk->rn;
    const uint64_t BATCH = 1ULL << 20, CH = 4096;
    if (n < (uint64_t)ORC_PAR_MIN_CHUNKS * CH) {
        /* a small block on the calling thread, candidate by candidate: the
         * team, the candidate lists and the in-order commit cost more than
         * its candidates */
        for (uint64_t a = 0; a < bk->ln; ++a) {
            if (op_is_unary(bk->op)) {
                if (process(s, bk->op, (int64_t)(bk->l0 + a), -1)) return 1;
                continue;
            }
            for (uint64_t b = 0; b < bk->rn; ++b)
                if (process(s, bk->op, (int64_t)(bk->l0 + a), (int64_t)(bk->r0 + b))) return 1;
        }
        return 0;
    }
    int nthreads = p->threads > 1 ? p->threads : 1;
    pend_t **lists = (pend_t **)calloc((BATCH + CH - 1) / CH, sizeof(pend_t *));
    uint32_t *lcount = (uint32_t *)calloc((BATCH + CH - 1) / CH, sizeof(uint32_t));
    int stop = 0;
    for (uint64_t base = 0; base < n && !stop; base += BATCH) {
        const uint64_t cnt = (n - base) < BATCH ? (n - base) : BATCH;
        const int64_t nch = (int64_t)((cnt + CH - 1) / CH);
        /* a batch of few chunks runs on the calling thread: starting the
         * team costs more than its candidates */
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads) if (nch >= ORC_PAR_MIN_CHUNKS)
        for (int64_t c = 0; c < nch; ++c) {
            uint64_t cs[ORC_MAX_TRACES];
            const uint64_t t0 = base + (uint64_t)c * CH;
            const uint64_t t1 = (t0 + CH < base + cnt) ? t0 + CH : base + cnt;
            pend_t *lst = lists[c];
            if (!lst) lst = lists[c] = (pend_t *)malloc(CH * sizeof(pend_t));
            uint32_t m = 0;
            for (uint64_t t = t0; t < t1; ++t) {
                const uint64_t a = op_is_unary(bk->op) ? bk->l0 + t : bk->l0 + t / bk->rn;
                const uint64_t b = op_is_unary(bk->op) ? 0 : bk->r0 + t % bk->rn;
                const uint64_t *lw = s->rows.cs + a * T;
                const uint64_t *rw = op_is_unary(bk->op) ? lw : s->rows.cs + b * T;
                for (int i = 0; i < T; ++i) cs[i] = apply_word(bk->op, lw[i], rw[i], p->len[i]);
                uint64_t h, l;
                make_key_s(p, s->S, cs, &h, &l);
                if (!kset_contains(&s->set, h, l)) {
                    lst[m].t = t;
                    lst[m].h = h;
                    lst[m].l = l;
                    ++m;
                }
            }
            lcount[c] = m;
        }
        /* in-order commit of the keys not seen before this batch */
        for (int64_t c = 0; c < nch && !stop; ++c) {
            for (uint32_t e = 0; e < lcount[c]; ++e) {
                const pend_t *pe = &lists[c][e];
                const uint64_t g = s->cands + pe->t;
                const int ins = kset_insert(&s->set, pe->h, pe->l);
                if (ins < 0) { s->error = ORC_LIMIT; stop = 1; break; }
                if (!ins) continue;
                const uint64_t a = op_is_unary(bk->op) ? bk->l0 + pe->t : bk->l0 + pe->t / bk->rn;
                const uint64_t b = op_is_unary(bk->op) ? 0 : bk->r0 + pe->t % bk->rn;
                if (s->rows.n >= p->max_rows || !rows_reserve(&s->rows, s->rows.n + 1)) {
                    s->error = ORC_LIMIT;
                    stop = 1;
                    break;
                }
                const uint64_t r = s->rows.n++;
                const uint64_t *lw = s->rows.cs + a * T;
                const uint64_t *rw = op_is_unary(bk->op) ? lw : s->rows.cs + b * T;
                uint64_t *cs = s->rows.cs + r * T;
                for (int i = 0; i < T; ++i) cs[i] = apply_word(bk->op, lw[i], rw[i], p->len[i]);
                s->rows.op[r] = (int8_t)bk->op;
                s->rows.left[r] = (int64_t)a;
                s->rows.right[r] = op_is_unary(bk->op) ? -1 : (int64_t)b;
                s->lvl_count[s->level]++;
                if (is_solution(p, cs)) {
                    s->found = 1;
                    s->found_row = (int64_t)r;
                    s->found_g = g;
                    s->cands += pe->t + 1;
                    stop = 2;
                    break;
                }
            }
        }
        if (stop == 2) break;
        if (!stop && base + cnt >= n) s->cands += n;
    }
    const int64_t nl = (int64_t)((BATCH + CH - 1) / CH);
    for (int64_t c = 0; c < nl; ++c) free(lists[c]);
    free(lists);
    free(lcount);
    return stop != 0;
}

static int level_parallel(search_t *s, int k) {
    for (int op = 0; op < 7; ++op) {
        if (op_is_unary(op)) {
            block_t bk = {op, s->lvl_start[k - 1], s->lvl_count[k - 1], 0, 0};
            if (bk.ln && run_block_parallel(s, &bk)) return 1;
            continue;
        }
        const int last = (op == OP_U) ? k - 2 : (k - 1) / 2;
        for (int i = 1; i <= last; ++i) {
            const int j = k - 1 - i;
            block_t bk = {op, s->lvl_start[i], s->lvl_count[i], s->lvl_start[j], s->lvl_count[j]};
            if (bk.ln && bk.rn && run_block_parallel(s, &bk)) return 1;
        }
    }
    return 0;
}

/* ----------------------------------------------------------- reconstruction */
static void rpn_of_row(const search_t *s, int64_t r, int16_t *out, int *n) {
    if (r < s->p->num_vars) {
        out[(*n)++] = (int16_t)r;
        return;
    }
    const int op = s->rows.op[r];
    rpn_of_row(s, s->rows.left[r], out, n);
    if (!op_is_unary(op)) rpn_of_row(s, s->rows.right[r], out, n);
    out[(*n)++] = (int16_t)(-(1 + op));
}

static double now_s(void) {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

static int check_problem(const orc_problem *p) {
    if (p->num_traces < 1 || p->num_traces > ORC_MAX_TRACES) return 0;
    if (p->num_vars < 1 || p->num_vars > ORC_MAX_VARS) return 0;
    if (p->num_pos < 0 || p->num_pos > p->num_traces) return 0;
    if (p->max_size < 1 || p->max_size > ORC_MAX_SIZE) return 0;
    if (p->rlx_type < 1 || p->rlx_type > 3) return 0;
    for (int i = 0; i < p->num_traces; ++i)
        if (p->len[i] < 1 || p->len[i] > 64) return 0;
    int unit = p->neg_type == 0 || p->neg_type == 1;
    if (p->neg_type < 0 || p->neg_type > 2) return 0;
    for (int i = 0; i < 8; ++i) {
        if (p->cost[i] < 0 || p->cost[i] > ORC_MAX_SIZE) return 0;
        if (p->cost[i] > 1) unit = 0;
    }
    if (!unit && (p->mode != ORC_MODE_CANONICAL || p->threads > 1)) return 0;
    if (atom_cost(p) > p->max_size) return 0;
    return 1;
}

/* The cached search; leaves its state in *sp for a following BS stage (the
 * caller frees it with search_free). */
static int run_search(const orc_problem *p, orc_result *res, search_t *sp) {
    search_t s;
    memset(&s, 0, sizeof(s));
    s.p = p;
    s.T = p->num_traces;
    s.S = len_sum(p);
    s.rows.T = s.T;
    s.tmp = (uint64_t *)malloc(s.T * sizeof(uint64_t));
    if (!kset_init(&s.set, 1 << 12) || !rows_reserve(&s.rows, (uint64_t)p->num_vars)) {
        res->status = ORC_LIMIT;
        goto done;
    }
    /* level 1: every proposition is a row (duplicates among them included),
     * its key enters the set, and each is tested as a size-1 solution in
     * proposition order (LTL_BS.cu:1127-1163, 1217). */
    const int c1 = atom_cost(p);
    s.level = c1;
    s.lvl_start[c1] = 0;
    trace_launch(&s, 1, 7, (uint64_t)p->num_vars);
    s.all_ltls = 0;
    for (int v = 0; v < p->num_vars; ++v) {
        s.all_ltls++;
        uint64_t *cs = s.rows.cs + (size_t)v * s.T;
        for (int i = 0; i < s.T; ++i) cs[i] = p->atoms[(size_t)v * s.T + i];
        s.rows.op[v] = OP_NONE;
        s.rows.left[v] = s.rows.right[v] = -1;
        s.rows.n++;
        uint64_t h, l;
        make_key_s(p, s.S, cs, &h, &l);
        kset_insert(&s.set, h, l);
        s.lvl_count[c1]++;
        s.cands++;
        if (is_solution(p, cs)) {
            s.found = 1;
            s.found_row = v;
            s.found_g = (uint64_t)v;
            break;
        }
    }
    for (int k = 1; k <= c1; ++k) s.lvl_start[k] = 0;
    res->level_rows[c1] = s.lvl_count[c1];
    res->level_cands[c1] = s.cands;
    res->size = c1;
    for (int k = c1 + 1; !s.found && k <= p->max_size; ++k) {
        s.level = k;
        s.cands = 0;
        s.lvl_start[k] = s.rows.n;
        s.lvl_count[k] = 0;
        if (p->mode == ORC_MODE_REFCOMPAT)
            level_refcompat(&s, k);
        else if (p->threads > 1)
            level_parallel(&s, k);
        else
            level_canonical(&s, k);
        res->level_rows[k] = s.lvl_count[k];
        res->level_cands[k] = s.cands;
        res->size = k;
        if (s.error) break;
    }
    if (s.error) {
        res->status = s.error;
    } else if (s.found) {
        res->status = ORC_FOUND;
        int n = 0;
        rpn_of_row(&s, s.found_row, res->rpn, &n);
        res->rpn_len = n;
        res->solution_index = s.found_g;
    } else {
        res->status = ORC_NOT_FOUND;
    }
    res->total_rows = s.rows.n;
    res->trace_len = s.trace_len;
done:
    *sp = s;
    return res->status;
}

static void search_free(search_t *s) {
    kset_free(&s->set);
    rows_free(&s->rows);
    free(s->tmp);
}

int orc_solve(const orc_problem *p, orc_result *res) {
    memset(res, 0, sizeof(*res));
    if (!check_problem(p)) return res->status = ORC_BAD_INPUT;
    const double t0 = now_s();
    search_t s;
    run_search(p, res, &s);
    search_free(&s);
    res->seconds = now_s() - t0;
    return res->status;
}

/* ------------------------------------------------------------------ BS stage
 * After a search that found nothing up to max_size, LTL_BS combines the cached
 * formulas with ~ & | over their step-0 vectors (BS LTL_BS.cu:870-1067):
 * every cached CS projects to a word with bit i = the formula holds at step 0
 * of trace i (transfer 808-822); a combination solves the sample when its word
 * is exactly the positive traces' bits (BSInsertInCache 279-288).  Restated
 * deterministically: the base entries of size c are the projections of the
 * level-c rows not seen earlier in canonical order; sizes c > max_size hold
 * ~ over size c-1, then & and | over size splits i <= (c-1)/2 (left index
 * major), each new word kept, the first solving candidate returned. */
typedef struct {
    uint64_t *v;
    int64_t *a, *b;
    int8_t *op;      /* -1: base entry, a = cache row */
    uint64_t n, cap;
} bsrows_t;

static int bs_push(bsrows_t *r, uint64_t v, int op, int64_t a, int64_t b) {
    if (r->n == r->cap) {
        uint64_t nc = r->cap ? 2 * r->cap : 1024;
        uint64_t *nv = (uint64_t *)realloc(r->v, nc * sizeof(uint64_t));
        if (!nv) return 0;
        r->v = nv;
        int64_t *na = (int64_t *)realloc(r->a, nc * sizeof(int64_t));
        if (!na) return 0;
        r->a = na;
        int64_t *nb = (int64_t *)realloc(r->b, nc * sizeof(int64_t));
        if (!nb) return 0;
        r->b = nb;
        int8_t *no = (int8_t *)realloc(r->op, nc);
        if (!no) return 0;
        r->op = no;
        r->cap = nc;
    }
    r->v[r->n] = v;
    r->op[r->n] = (int8_t)op;
    r->a[r->n] = a;
    r->b[r->n] = b;
    r->n++;
    return 1;
}

static void bs_rpn(const search_t *s, const bsrows_t *r, int64_t e, int16_t *out, int *n) {
    if (r->op[e] < 0) {
        rpn_of_row(s, r->a[e], out, n);
        return;
    }
    bs_rpn(s, r, r->a[e], out, n);
    if (r->op[e] != OP_NOT) bs_rpn(s, r, r->b[e], out, n);
    out[(*n)++] = (int16_t)(-(1 + r->op[e]));
}

static int bs_stage(search_t *s, int bs_max, orc_result *res) {
    const orc_problem *p = s->p;
    const int T = s->T, K = p->max_size;
    if (T > 64) return ORC_LIMIT;
    const uint64_t full = T == 64 ? ~0ULL : ((1ULL << T) - 1);
    const uint64_t target = p->num_pos == 64 ? ~0ULL : ((1ULL << p->num_pos) - 1);
    uint64_t st[ORC_MAX_SIZE + 2], cn[ORC_MAX_SIZE + 2];
    memset(st, 0, sizeof(st));
    memset(cn, 0, sizeof(cn));
    bsrows_t r;
    memset(&r, 0, sizeof(r));
    kset set;
    int status = ORC_NOT_FOUND;
    if (!kset_init(&set, 1 << 12)) return ORC_LIMIT;
    for (int c = 1; c <= K; ++c) {
        st[c] = r.n;
        for (uint64_t i = 0; i < s->lvl_count[c]; ++i) {
            const int64_t row = (int64_t)(s->lvl_start[c] + i);
            const uint64_t *cs = row_cs(s, row);
            uint64_t v = 0;
            for (int t = 0; t < T; ++t) v |= (cs[t] & 1ULL) << t;
            const int ins = kset_insert(&set, v & 0xffffffffULL, v >> 32);
            if (ins < 0 || (ins && !bs_push(&r, v, -1, row, -1))) { status = ORC_LIMIT; goto out; }
        }
        cn[c] = r.n - st[c];
    }
    for (int c = K + 1; c <= bs_max; ++c) {
        st[c] = r.n;
        uint64_t cands = 0;
        int64_t win = -1;
        int wop = 0;
        int64_t wa = -1, wb = -1;
        for (int op = 0; op < 3 && win < 0; ++op) {
            if (op == OP_NOT) {
                for (uint64_t a = 0; a < cn[c - 1] && win < 0; ++a) {
                    const int64_t ea = (int64_t)(st[c - 1] + a);
                    const uint64_t v = ~r.v[ea] & full;
                    ++cands;
                    if (v == target) { win = (int64_t)cands - 1; wop = op; wa = ea; break; }
                    const int ins = kset_insert(&set, v & 0xffffffffULL, v >> 32);
                    if (ins < 0 || (ins && !bs_push(&r, v, op, ea, -1))) { status = ORC_LIMIT; goto out; }
                }
                continue;
            }
            for (int i = 1; 2 * i <= c - 1 && win < 0; ++i) {
                const int j = c - 1 - i;
                for (uint64_t a = 0; a < cn[i] && win < 0; ++a)
                    for (uint64_t b = 0; b < cn[j]; ++b) {
                        const int64_t ea = (int64_t)(st[i] + a), eb = (int64_t)(st[j] + b);
                        const uint64_t v = op == OP_AND ? (r.v[ea] & r.v[eb]) : (r.v[ea] | r.v[eb]);
                        ++cands;
                        if (v == target) { win = (int64_t)cands - 1; wop = op; wa = ea; wb = eb; break; }
                        const int ins = kset_insert(&set, v & 0xffffffffULL, v >> 32);
                        if (ins < 0 || (ins && !bs_push(&r, v, op, ea, eb))) { status = ORC_LIMIT; goto out; }
                    }
            }
        }
        cn[c] = r.n - st[c];
        res->level_rows[c] = cn[c];
        res->level_cands[c] = cands;
        res->size = c;
        if (win >= 0) {
            res->level_rows[c] = cn[c] + 1;
            if (!bs_push(&r, target, wop, wa, wb)) { status = ORC_LIMIT; goto out; }
            int n = 0;
            bs_rpn(s, &r, (int64_t)r.n - 1, res->rpn, &n);
            res->rpn_len = n;
            res->solution_index = (uint64_t)win;
            status = ORC_FOUND;
            break;
        }
    }
out:
    res->total_rows = s->rows.n;
    for (int c = K + 1; c <= res->size; ++c) res->total_rows += res->level_rows[c];
    kset_free(&set);
    free(r.v);
    free(r.a);
    free(r.b);
    free(r.op);
    return status;
}

int orc_solve_bs(const orc_problem *p, int bs_max, orc_result *res) {
    memset(res, 0, sizeof(*res));
    if (!check_problem(p) || bs_max > ORC_MAX_SIZE) return res->status = ORC_BAD_INPUT;
    for (int i = 0; i < 8; ++i)
        if (p->cost[i] > 1) return res->status = ORC_BAD_INPUT;   /* the BS stage uses unit costs */
    const double t0 = now_s();
    search_t s;
    run_search(p, res, &s);
    if (res->status == ORC_NOT_FOUND && bs_max > p->max_size && p->mode == ORC_MODE_CANONICAL)
        res->status = bs_stage(&s, bs_max, res);
    search_free(&s);
    res->seconds = now_s() - t0;
    return res->status;
}

/* ---------------------------------------------------- RPN evaluation (nocache) */
int orc_eval_rpn(const orc_problem *p, const int16_t *rpn, int rpn_len, uint64_t *cs_out) {
    uint64_t st[ORC_MAX_SIZE + 1];
    int sol = 1;
    for (int i = 0; i < p->num_traces; ++i) {
        int sp = 0;
        for (int j = 0; j < rpn_len; ++j) {
            const int tk = rpn[j];
            if (tk >= 0) {
                if (tk >= p->num_vars || sp > ORC_MAX_SIZE) return -1;
                st[sp++] = p->atoms[(size_t)tk * p->num_traces + i];
                continue;
            }
            const int op = -tk - 1;
            if (op < 0 || op > 6) return -1;
            if (op_is_unary(op)) {
                if (sp < 1) return -1;
                st[sp - 1] = apply_word(op, st[sp - 1], 0, p->len[i]);
            } else {
                if (sp < 2) return -1;
                st[sp - 2] = apply_word(op, st[sp - 2], st[sp - 1], p->len[i]);
                --sp;
            }
        }
        if (sp != 1) return -1;
        if (cs_out) cs_out[i] = st[0];
        const int bit = (int)(st[0] & 1);
        if ((i < p->num_pos) != (bit == 1)) sol = 0;
    }
    return sol;
}

/* ------------------------------------- exhaustive nocache-order enumeration */
typedef unsigned __int128 u128;

static void decode_number(u128 n, int size, const u128 (*cnt)[8], int16_t *out, int *len) {
    if (size == 1) {
        out[(*len)++] = (int16_t)n;
        return;
    }
    int op = 0;
    while (n >= cnt[size][op]) n -= cnt[size][op++];
    const int sub = size - 1;
    if (op_is_unary(op)) {
        decode_number(n, sub, cnt, out, len);
    } else {
        int left = 1;
        while (n >= cnt[left][7] * cnt[sub - left][7]) {
            n -= cnt[left][7] * cnt[sub - left][7];
            ++left;
        }
        const u128 nr = cnt[sub - left][7];
        decode_number(n / nr, left, cnt, out, len);
        decode_number(n % nr, sub - left, cnt, out, len);
    }
    out[(*len)++] = (int16_t)(-(1 + op));
}

int orc_exhaustive(const orc_problem *p, uint64_t max_formulas, orc_result *res) {
    memset(res, 0, sizeof(*res));
    if (!check_problem(p)) return res->status = ORC_BAD_INPUT;
    const double t0 = now_s();
    static u128 cnt[ORC_MAX_SIZE + 1][8];
    memset(cnt, 0, sizeof(cnt));
    const int A = p->num_vars, K = p->max_size;
    cnt[1][7] = (u128)A;
    if (K >= 2) {
        cnt[2][0] = cnt[2][3] = cnt[2][4] = cnt[2][5] = (u128)A;
        cnt[2][7] = (u128)(4 * A);
    }
    for (int i = 3; i <= K; ++i) {
        u128 un = cnt[i - 1][7], com = 0, ncom = 0;
        for (int j = 1; j <= (i - 1) / 2; ++j) com += cnt[j][7] * cnt[i - j - 1][7];
        for (int j = 1; j <= i - 2; ++j) ncom += cnt[j][7] * cnt[i - j - 1][7];
        cnt[i][0] = cnt[i][3] = cnt[i][4] = cnt[i][5] = un;
        cnt[i][1] = cnt[i][2] = com;
        cnt[i][6] = ncom;
        cnt[i][7] = 4 * un + 2 * com + ncom;
    }
    uint64_t evaluated = 0;
    for (int k = 1; k <= K; ++k) {
        res->size = k;
        for (u128 n = 0; n < cnt[k][7]; ++n) {
            if (evaluated >= max_formulas) {
                res->status = ORC_LIMIT;
                goto out;
            }
            ++evaluated;
            res->level_cands[k]++;
            int16_t rpn[ORC_MAX_SIZE];
            int len = 0;
            decode_number(n, k, (const u128(*)[8])cnt, rpn, &len);
            if (orc_eval_rpn(p, rpn, len, NULL) == 1) {
                memcpy(res->rpn, rpn, len * sizeof(int16_t));
                res->rpn_len = len;
                res->solution_index = (uint64_t)n;
                res->status = ORC_FOUND;
                goto out;
            }
        }
    }
    res->status = ORC_NOT_FOUND;
out:
    res->seconds = now_s() - t0;
    (void)OPCH;
    return res->status;
}
