/*
 * oracle.c — CPU restatement of the reference's operator semantics.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py load this file's library, as the checker or
 * as the timed CPU stand-in for the reference's own CPU path; the product
 * never does.
 *
 * Every function follows crates/oxidelake-device/src/cpu/kernels.rs of the
 * reference (cited per function).  Built with -ffp-contract=off and without
 * -ffast-math, so float arithmetic is the reference's: one IEEE operation per
 * Rust operator, no fused multiply-add, sums folded in index order.
 */
#include "oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------ */
/* small helpers                                                            */
/* ------------------------------------------------------------------------ */

static inline int is_valid(const orc_column* c, int64_t i) {
    return c->validity == NULL ? 1 : (c->validity[i >> 3] >> (i & 7)) & 1;
}
static inline int64_t get_i64(const orc_column* c, int64_t i) {
    return ((const int64_t*)c->values)[i];
}
static inline int32_t get_i32(const orc_column* c, int64_t i) {
    return ((const int32_t*)c->values)[i];
}
static inline double get_f64(const orc_column* c, int64_t i) {
    return ((const double*)c->values)[i];
}
static inline uint64_t f64_bits(double x) {
    uint64_t b;
    memcpy(&b, &x, 8);
    return b;
}
static inline double bits_f64(uint64_t b) {
    double x;
    memcpy(&x, &b, 8);
    return x;
}
static inline uint32_t f32_bits(float x) {
    uint32_t b;
    memcpy(&b, &x, 4);
    return b;
}

/* total_order_key, cpu/kernels.rs:825-830: flip every bit but the sign of a
 * negative value, so comparing keys as int64 is f64::total_cmp. */
int64_t orc_total_order_key(double x) {
    int64_t bits = (int64_t)f64_bits(x);
    return bits ^ (int64_t)(((uint64_t)(bits >> 63)) >> 1);
}

/* from_total_order_key, cpu/kernels.rs:836-838: the transform is an involution. */
double orc_from_total_order_key(int64_t key) {
    return bits_f64((uint64_t)(key ^ (int64_t)(((uint64_t)(key >> 63)) >> 1)));
}

/* The order a Float64 filter compares in: positive_zero (cpu/kernels.rs:62-69)
 * then IEEE totalOrder (the arrow cmp kernels evaluate_predicate calls,
 * cpu/kernels.rs:99-141). */
int64_t orc_filter_order_key(double x) {
    if (f64_bits(x) == 0x8000000000000000ULL) x = 0.0;
    return orc_total_order_key(x);
}

/* slot_hash, crates/oxidelake-device/src/join_slots.rs:36-45 (murmur3 fmix64). */
uint32_t orc_slot_hash(int64_t key, uint32_t capacity) {
    uint64_t h = (uint64_t)key;
    h ^= h >> 33;
    h *= 0xff51afd7ed558ccdULL;
    h ^= h >> 33;
    h *= 0xc4ceb9fe1a85ec53ULL;
    h ^= h >> 33;
    return (uint32_t)(h & (uint64_t)(capacity - 1u));
}

/* l2, cpu/kernels.rs:909-915: Σ (x−y)² folded in index order from −0.0
 * (Rust's f32 Sum), then sqrt. */
float orc_l2(const float* a, const float* b, int64_t dim) {
    float s = -0.0f;
    for (int64_t i = 0; i < dim; i++) {
        float d = a[i] - b[i];
        float sq = d * d;
        s = s + sq;
    }
    return sqrtf(s);
}

/* cosine, cpu/kernels.rs:918-927: 1 − dot/(na·nb), NaN when a norm is 0. */
float orc_cosine(const float* a, const float* b, int64_t dim) {
    float dot = -0.0f, sa = -0.0f, sb = -0.0f;
    for (int64_t i = 0; i < dim; i++) {
        float p = a[i] * b[i];
        dot = dot + p;
    }
    for (int64_t i = 0; i < dim; i++) {
        float p = a[i] * a[i];
        sa = sa + p;
    }
    for (int64_t i = 0; i < dim; i++) {
        float p = b[i] * b[i];
        sb = sb + p;
    }
    float na = sqrtf(sa), nb = sqrtf(sb);
    if (na == 0.0f || nb == 0.0f) return NAN;
    float den = na * nb;
    float q = dot / den;
    return 1.0f - q;
}

/* ------------------------------------------------------------------------ */
/* int64 -> int64 open-addressing map (test-side HashMap)                   */
/* ------------------------------------------------------------------------ */

typedef struct imap {
    int64_t* keys;
    int64_t* vals;
    uint8_t* used;
    uint64_t cap;
    uint64_t len;
} imap;

static uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

static int imap_init(imap* m, uint64_t expect) {
    uint64_t cap = 16;
    while (cap < expect * 2) cap <<= 1;
    m->keys = (int64_t*)malloc(cap * 8);
    m->vals = (int64_t*)malloc(cap * 8);
    m->used = (uint8_t*)calloc(cap, 1);
    m->cap = cap;
    m->len = 0;
    return (m->keys && m->vals && m->used) ? 0 : -1;
}
static void imap_free(imap* m) {
    free(m->keys);
    free(m->vals);
    free(m->used);
    memset(m, 0, sizeof *m);
}
static int64_t* imap_find(const imap* m, int64_t key) {
    uint64_t s = mix64((uint64_t)key) & (m->cap - 1);
    while (m->used[s]) {
        if (m->keys[s] == key) return &m->vals[s];
        s = (s + 1) & (m->cap - 1);
    }
    return NULL;
}
static int imap_grow(imap* m) {
    imap n;
    if (imap_init(&n, m->cap) != 0) return -1;
    for (uint64_t s = 0; s < m->cap; s++) {
        if (!m->used[s]) continue;
        uint64_t t = mix64((uint64_t)m->keys[s]) & (n.cap - 1);
        while (n.used[t]) t = (t + 1) & (n.cap - 1);
        n.used[t] = 1;
        n.keys[t] = m->keys[s];
        n.vals[t] = m->vals[s];
        n.len++;
    }
    imap_free(m);
    *m = n;
    return 0;
}
/* Returns the value slot for key, inserting `fresh` when absent (*inserted = 1). */
static int64_t* imap_entry(imap* m, int64_t key, int64_t fresh, int* inserted) {
    if ((m->len + 1) * 2 > m->cap) imap_grow(m);
    uint64_t s = mix64((uint64_t)key) & (m->cap - 1);
    while (m->used[s]) {
        if (m->keys[s] == key) {
            *inserted = 0;
            return &m->vals[s];
        }
        s = (s + 1) & (m->cap - 1);
    }
    m->used[s] = 1;
    m->keys[s] = key;
    m->vals[s] = fresh;
    m->len++;
    *inserted = 1;
    return &m->vals[s];
}

/* ------------------------------------------------------------------------ */
/* filter                                                                   */
/* ------------------------------------------------------------------------ */

static int leaf_types_ok(const orc_column* cols, int32_t ncols, const orc_leaf* leaves,
                         int32_t nleaves) {
    for (int32_t l = 0; l < nleaves; l++) {
        if (leaves[l].column < 0 || leaves[l].column >= ncols) return ORC_ERR_PLAN;
        int32_t t = cols[leaves[l].column].type;
        /* cpu/kernels.rs:110-119: the literal's type must be the column's. */
        if (t != leaves[l].lit_type) return ORC_ERR_UNSUPPORTED;
        if (t != ORC_INT64 && t != ORC_FLOAT64 && t != ORC_INT32) return ORC_ERR_UNSUPPORTED;
    }
    return ORC_OK;
}

static inline int cmp_result(int op, int c /* -1, 0, 1 */) {
    switch (op) {
        case ORC_EQ: return c == 0;
        case ORC_LT: return c < 0;
        case ORC_LTEQ: return c <= 0;
        case ORC_GT: return c > 0;
        default: return c >= 0;
    }
}

/* One leaf at one row: NULL operand → not selected (a NULL mask entry drops
 * the row, cpu/kernels.rs:4-6 and filter_record_batch). */
static inline int leaf_true(const orc_column* cols, const orc_leaf* lf, int64_t row) {
    const orc_column* c = &cols[lf->column];
    if (!is_valid(c, row)) return 0;
    int cmp;
    if (c->type == ORC_FLOAT64) {
        int64_t a = orc_filter_order_key(get_f64(c, row));
        int64_t b = orc_filter_order_key(lf->lit.f);
        cmp = (a > b) - (a < b);
    } else {
        int64_t a = c->type == ORC_INT64 ? get_i64(c, row) : (int64_t)get_i32(c, row);
        int64_t b = lf->lit.i;
        cmp = (a > b) - (a < b);
    }
    return cmp_result(lf->op, cmp);
}

static inline int row_selected(const orc_column* cols, const orc_leaf* leaves, int32_t nleaves,
                               int64_t row) {
    for (int32_t l = 0; l < nleaves; l++)
        if (!leaf_true(cols, &leaves[l], row)) return 0;
    return 1;
}

/* evaluate_predicate + filter_project, cpu/kernels.rs:99-152: the rows the
 * mask keeps, in row order (projection is a gather of these rows). */
int64_t orc_filter(const orc_column* cols, int32_t ncols, const orc_leaf* leaves, int32_t nleaves,
                   uint32_t* out_rows) {
    int rc = leaf_types_ok(cols, ncols, leaves, nleaves);
    if (rc != ORC_OK) return rc;
    int64_t n = ncols > 0 ? cols[0].length : 0;
    int64_t k = 0;
    for (int64_t i = 0; i < n; i++)
        if (row_selected(cols, leaves, nleaves, i)) out_rows[k++] = (uint32_t)i;
    return k;
}

/* ------------------------------------------------------------------------ */
/* join                                                                     */
/* ------------------------------------------------------------------------ */

struct orc_join_table {
    imap ranges;        /* key -> index into run arrays */
    int64_t ndistinct;
    int64_t* run_keys;
    uint32_t* run_start;
    uint32_t* run_count;
    uint32_t* rows;
    int64_t nrows;
};

/* JoinTable::build, cpu/kernels.rs:199-226: NULL keys skipped; one run per
 * distinct key into a row array grouped by key, build order within a key.
 * (Runs are numbered here in first-seen order; the reference's HashMap
 * order is arbitrary and invisible in any output.) */
int32_t orc_join_build(const orc_column* key, orc_join_table** out) {
    if (key->type != ORC_INT64 && key->type != ORC_INT32) return ORC_ERR_UNSUPPORTED;
    int64_t n = key->length;
    orc_join_table* t = (orc_join_table*)calloc(1, sizeof *t);
    imap_init(&t->ranges, 16);
    int64_t cap = 16;
    t->run_keys = (int64_t*)malloc(cap * 8);
    t->run_count = (uint32_t*)malloc(cap * 4);
    for (int64_t i = 0; i < n; i++) {
        if (!is_valid(key, i)) continue;
        int64_t k = key->type == ORC_INT64 ? get_i64(key, i) : get_i32(key, i);
        int ins;
        int64_t* v = imap_entry(&t->ranges, k, t->ndistinct, &ins);
        if (ins) {
            if (t->ndistinct == cap) {
                cap *= 2;
                t->run_keys = (int64_t*)realloc(t->run_keys, cap * 8);
                t->run_count = (uint32_t*)realloc(t->run_count, cap * 4);
            }
            t->run_keys[t->ndistinct] = k;
            t->run_count[t->ndistinct] = 0;
            t->ndistinct++;
        }
        t->run_count[*v]++;
        t->nrows++;
    }
    t->run_start = (uint32_t*)malloc((t->ndistinct + 1) * 4);
    uint32_t next = 0;
    for (int64_t r = 0; r < t->ndistinct; r++) {
        t->run_start[r] = next;
        next += t->run_count[r];
    }
    uint32_t* cursor = (uint32_t*)malloc((t->ndistinct + 1) * 4);
    memcpy(cursor, t->run_start, t->ndistinct * 4);
    t->rows = (uint32_t*)malloc((t->nrows + 1) * 4);
    for (int64_t i = 0; i < n; i++) {
        if (!is_valid(key, i)) continue;
        int64_t k = key->type == ORC_INT64 ? get_i64(key, i) : get_i32(key, i);
        int64_t r = *imap_find(&t->ranges, k);
        t->rows[cursor[r]++] = (uint32_t)i;
    }
    free(cursor);
    *out = t;
    return ORC_OK;
}

void orc_join_free(orc_join_table* t) {
    if (!t) return;
    imap_free(&t->ranges);
    free(t->run_keys);
    free(t->run_start);
    free(t->run_count);
    free(t->rows);
    free(t);
}
int64_t orc_join_distinct(const orc_join_table* t) { return t->ndistinct; }
int64_t orc_join_nrows(const orc_join_table* t) { return t->nrows; }
void orc_join_export(const orc_join_table* t, int64_t* keys, uint32_t* starts, uint32_t* counts,
                     uint32_t* rows) {
    memcpy(keys, t->run_keys, t->ndistinct * 8);
    memcpy(starts, t->run_start, t->ndistinct * 4);
    memcpy(counts, t->run_count, t->ndistinct * 4);
    memcpy(rows, t->rows, t->nrows * 4);
}

static inline int join_run(const orc_join_table* t, int64_t key, uint32_t* start, uint32_t* count) {
    const int64_t* r = imap_find(&t->ranges, key);
    if (!r) return 0;
    *start = t->run_start[*r];
    *count = t->run_count[*r];
    return 1;
}

/* JoinMatches::probe, cpu/kernels.rs:323-342. */
int64_t orc_join_probe(const orc_join_table* t, const orc_column* key, uint64_t* offsets,
                       uint32_t* starts) {
    uint64_t total = 0;
    for (int64_t i = 0; i < key->length; i++) {
        offsets[i] = total;
        uint32_t s = 0, c = 0;
        if (is_valid(key, i)) {
            int64_t k = key->type == ORC_INT64 ? get_i64(key, i) : get_i32(key, i);
            if (!join_run(t, k, &s, &c)) s = c = 0;
        }
        starts[i] = s;
        total += c;
    }
    offsets[key->length] = total;
    return (int64_t)total;
}

/* JoinMatches::pairs, cpu/kernels.rs:360-406. */
int32_t orc_join_pairs(const orc_join_table* t, const uint64_t* offsets, const uint32_t* starts,
                       int64_t nprobe, uint64_t first, uint64_t rows, uint32_t* left,
                       uint32_t* right) {
    uint64_t total = offsets[nprobe];
    if (first + rows < first || first + rows > total) return ORC_ERR_EXECUTION;
    uint64_t end = first + rows;
    /* partition_point(offset <= first) - 1 */
    int64_t lo = 0, hi = nprobe + 1;
    while (lo < hi) {
        int64_t mid = lo + (hi - lo) / 2;
        if (offsets[mid] <= first) lo = mid + 1;
        else hi = mid;
    }
    int64_t row = lo > 0 ? lo - 1 : 0;
    uint64_t at = first, w = 0;
    while (at < end) {
        uint64_t a = offsets[row], b = offsets[row + 1];
        uint64_t upto = b < end ? b : end;
        if (upto > at) {
            uint64_t s = starts[row];
            for (uint64_t m = at; m < upto; m++) {
                uint64_t idx = s + (m - a);
                if (idx >= (uint64_t)t->nrows) return ORC_ERR_EXECUTION;
                left[w] = (uint32_t)row;
                right[w] = t->rows[idx];
                w++;
            }
            at = upto;
        }
        row++;
    }
    return ORC_OK;
}

/* ------------------------------------------------------------------------ */
/* grouped aggregation                                                      */
/* ------------------------------------------------------------------------ */

typedef struct agg_state {
    int32_t func;
    int32_t in_type;
    int64_t* ival;  /* SUM int / MIN / MAX int, COUNT */
    double* dval;   /* SUM f64 / AVG sum / MIN / MAX f64 */
    uint64_t* cnt;  /* non-NULL values seen (SUM/MIN/MAX/AVG), rows (COUNT*) */
} agg_state;

struct orc_agg {
    int32_t group_by;
    int32_t key_type;
    int32_t n;
    int32_t columns[ORC_MAX_AGGREGATES];
    agg_state st[ORC_MAX_AGGREGATES];
    imap index;
    int64_t null_group;
    int64_t ngroups;
    int64_t cap;
    int64_t* keys;
    uint8_t* key_valid;
};

static int agg_type_ok(int32_t func, int32_t t) {
    switch (func) {
        case ORC_COUNT_STAR: return 1;
        case ORC_COUNT: return t == ORC_INT64 || t == ORC_FLOAT64 || t == ORC_INT32;
        case ORC_SUM:
        case ORC_MIN:
        case ORC_MAX:
        case ORC_AVG: return t == ORC_INT64 || t == ORC_FLOAT64 || t == ORC_INT32;
        default: return 0;
    }
}

/* GroupedAggregator::new, cpu/kernels.rs:693-730 (types checked up front). */
int32_t orc_agg_new(const orc_column* cols, int32_t ncols, const orc_agg_spec* spec,
                    orc_agg** out) {
    if (spec->group_by < 0 || spec->group_by >= ncols) return ORC_ERR_PLAN;
    int32_t kt = cols[spec->group_by].type;
    if (kt != ORC_INT64 && kt != ORC_INT32) return ORC_ERR_UNSUPPORTED;
    if (spec->naggregates < 0 || spec->naggregates > ORC_MAX_AGGREGATES) return ORC_ERR_PLAN;
    orc_agg* a = (orc_agg*)calloc(1, sizeof *a);
    a->group_by = spec->group_by;
    a->key_type = kt;
    a->n = spec->naggregates;
    for (int32_t j = 0; j < a->n; j++) {
        int32_t f = spec->funcs[j], c = spec->columns[j];
        int32_t t = ORC_INT64;
        if (f != ORC_COUNT_STAR) {
            if (c < 0 || c >= ncols) {
                free(a);
                return ORC_ERR_PLAN;
            }
            t = cols[c].type;
        }
        if (!agg_type_ok(f, t)) {
            free(a);
            return ORC_ERR_UNSUPPORTED;
        }
        a->columns[j] = c;
        a->st[j].func = f;
        a->st[j].in_type = t;
    }
    imap_init(&a->index, 16);
    a->null_group = -1;
    return ORC_OK + (*out = a, 0);
}

static void agg_grow(orc_agg* a, int64_t need) {
    if (need <= a->cap) return;
    int64_t cap = a->cap ? a->cap : 16;
    while (cap < need) cap *= 2;
    a->keys = (int64_t*)realloc(a->keys, cap * 8);
    a->key_valid = (uint8_t*)realloc(a->key_valid, cap);
    for (int32_t j = 0; j < a->n; j++) {
        agg_state* s = &a->st[j];
        s->ival = (int64_t*)realloc(s->ival, cap * 8);
        s->dval = (double*)realloc(s->dval, cap * 8);
        s->cnt = (uint64_t*)realloc(s->cnt, cap * 8);
    }
    a->cap = cap;
}

/* group_ids, cpu/kernels.rs:738-762: first-seen numbering, NULL its own group. */
static int64_t agg_group(orc_agg* a, int valid, int64_t key) {
    int64_t g;
    if (!valid) {
        if (a->null_group >= 0) return a->null_group;
        g = a->ngroups;
        a->null_group = g;
    } else {
        int ins;
        int64_t* v = imap_entry(&a->index, key, a->ngroups, &ins);
        if (!ins) return *v;
        g = a->ngroups;
    }
    agg_grow(a, g + 1);
    a->keys[g] = valid ? key : 0;
    a->key_valid[g] = (uint8_t)valid;
    for (int32_t j = 0; j < a->n; j++) {
        a->st[j].ival[g] = 0;
        a->st[j].dval[g] = 0.0;
        a->st[j].cnt[g] = 0;
    }
    a->ngroups++;
    return g;
}

/* total_min / total_max, cpu/kernels.rs:531-538. */
static inline double total_min(double held, double v) {
    return orc_total_order_key(v) < orc_total_order_key(held) ? v : held;
}
static inline double total_max(double held, double v) {
    return orc_total_order_key(v) > orc_total_order_key(held) ? v : held;
}

/* Accumulator::update for one value, cpu/kernels.rs:572-629 (fold with
 * `first` / `next`).  is_f: the value is a double in dv, else an integer in iv. */
static inline void agg_fold(agg_state* s, int64_t g, int is_f, int64_t iv, double dv) {
    uint64_t seen = s->cnt[g];
    switch (s->func) {
        case ORC_SUM:
            if (is_f) s->dval[g] = seen ? s->dval[g] + dv : 0.0 + dv;
            else s->ival[g] = seen ? (int64_t)((uint64_t)s->ival[g] + (uint64_t)iv) : iv;
            break;
        case ORC_AVG:
            /* AVG: DataFusion casts an integer input to Float64; sum / count. */
            if (!is_f) dv = (double)iv;
            s->dval[g] = seen ? s->dval[g] + dv : 0.0 + dv;
            break;
        case ORC_MIN:
            if (is_f) s->dval[g] = seen ? total_min(s->dval[g], dv) : dv;
            else s->ival[g] = seen ? (iv < s->ival[g] ? iv : s->ival[g]) : iv;
            break;
        case ORC_MAX:
            if (is_f) s->dval[g] = seen ? total_max(s->dval[g], dv) : dv;
            else s->ival[g] = seen ? (iv > s->ival[g] ? iv : s->ival[g]) : iv;
            break;
        default: break;
    }
    s->cnt[g] = seen + 1;
}

static inline void agg_update_row(orc_agg* a, const orc_column* cols, int64_t g, int64_t row) {
    for (int32_t j = 0; j < a->n; j++) {
        agg_state* s = &a->st[j];
        if (s->func == ORC_COUNT_STAR) {
            s->cnt[g]++;
            continue;
        }
        const orc_column* c = &cols[a->columns[j]];
        if (!is_valid(c, row)) continue;
        if (s->func == ORC_COUNT) {
            s->cnt[g]++;
            continue;
        }
        if (c->type == ORC_FLOAT64) agg_fold(s, g, 1, 0, get_f64(c, row));
        else if (c->type == ORC_INT64) agg_fold(s, g, 0, get_i64(c, row), 0.0);
        else agg_fold(s, g, 0, get_i32(c, row), 0.0);
    }
}

static inline int64_t key_at(const orc_column* k, int64_t row) {
    return k->type == ORC_INT64 ? get_i64(k, row) : (int64_t)get_i32(k, row);
}

/* GroupedAggregator::update, cpu/kernels.rs:765-772, over the rows a fused
 * WHERE keeps (filter_project then aggregate). */
int32_t orc_agg_update(orc_agg* a, const orc_column* cols, int32_t ncols, const orc_leaf* leaves,
                       int32_t nleaves) {
    int rc = leaf_types_ok(cols, ncols, leaves, nleaves);
    if (rc != ORC_OK) return rc;
    const orc_column* k = &cols[a->group_by];
    for (int64_t row = 0; row < k->length; row++) {
        if (!row_selected(cols, leaves, nleaves, row)) continue;
        int v = is_valid(k, row);
        int64_t g = agg_group(a, v, v ? key_at(k, row) : 0);
        agg_update_row(a, cols, g, row);
    }
    return ORC_OK;
}

/* GroupedAggregator::merge + Accumulator::merge, cpu/kernels.rs:634-645,
 * 776-790: COUNT partials add, the others refold like input. */
int32_t orc_agg_merge(orc_agg* a, const orc_column* partial, int32_t ncols) {
    if (ncols != 1 + a->n) return ORC_ERR_EXECUTION;
    const orc_column* k = &partial[0];
    for (int32_t j = 0; j < a->n; j++)
        if (a->st[j].func == ORC_AVG) return ORC_ERR_UNSUPPORTED;
    for (int64_t row = 0; row < k->length; row++) {
        int v = is_valid(k, row);
        int64_t g = agg_group(a, v, v ? key_at(k, row) : 0);
        for (int32_t j = 0; j < a->n; j++) {
            agg_state* s = &a->st[j];
            const orc_column* c = &partial[1 + j];
            if (!is_valid(c, row)) continue;
            if (s->func == ORC_COUNT || s->func == ORC_COUNT_STAR) {
                s->cnt[g] = s->cnt[g] + (uint64_t)get_i64(c, row);
                continue;
            }
            if (c->type == ORC_FLOAT64) agg_fold(s, g, 1, 0, get_f64(c, row));
            else if (c->type == ORC_INT64) agg_fold(s, g, 0, get_i64(c, row), 0.0);
            else agg_fold(s, g, 0, get_i32(c, row), 0.0);
        }
    }
    return ORC_OK;
}

int64_t orc_agg_groups(const orc_agg* a) { return a->ngroups; }

static const orc_agg* g_sort_agg;
static int cmp_groups(const void* x, const void* y) {
    int64_t i = *(const int64_t*)x, j = *(const int64_t*)y;
    const orc_agg* a = g_sort_agg;
    int ni = !a->key_valid[i], nj = !a->key_valid[j];
    if (ni != nj) return ni - nj; /* NULL last */
    if (ni) return 0;
    return (a->keys[i] > a->keys[j]) - (a->keys[i] < a->keys[j]);
}

/* GroupedAggregator::finish + Accumulator::finish, cpu/kernels.rs:648-666,
 * 793-811: groups sorted by key with NULL last; SUM/MIN/MAX NULL for a
 * group with no values; COUNT never NULL. */
void orc_agg_finish(const orc_agg* a, int64_t* keys, uint8_t* key_valid, int64_t* values,
                    uint8_t* valid) {
    int64_t G = a->ngroups;
    int64_t* order = (int64_t*)malloc((G + 1) * 8);
    for (int64_t g = 0; g < G; g++) order[g] = g;
    g_sort_agg = a;
    qsort(order, (size_t)G, 8, cmp_groups);
    for (int64_t r = 0; r < G; r++) {
        int64_t g = order[r];
        keys[r] = a->keys[g];
        key_valid[r] = a->key_valid[g];
        for (int32_t j = 0; j < a->n; j++) {
            const agg_state* s = &a->st[j];
            int64_t* out = &values[j * G + r];
            uint8_t* ok = &valid[j * G + r];
            switch (s->func) {
                case ORC_COUNT:
                case ORC_COUNT_STAR:
                    *out = (int64_t)s->cnt[g];
                    *ok = 1;
                    break;
                case ORC_AVG: {
                    *ok = s->cnt[g] > 0;
                    double q = s->cnt[g] ? s->dval[g] / (double)s->cnt[g] : 0.0;
                    *out = (int64_t)f64_bits(q);
                    break;
                }
                default:
                    *ok = s->cnt[g] > 0;
                    if (s->in_type == ORC_FLOAT64)
                        *out = (int64_t)f64_bits(s->cnt[g] ? s->dval[g] : 0.0);
                    else *out = s->cnt[g] ? s->ival[g] : 0;
                    break;
            }
        }
    }
    free(order);
}

void orc_agg_free(orc_agg* a) {
    if (!a) return;
    imap_free(&a->index);
    free(a->keys);
    free(a->key_valid);
    for (int32_t j = 0; j < a->n; j++) {
        free(a->st[j].ival);
        free(a->st[j].dval);
        free(a->st[j].cnt);
    }
    free(a);
}

/* Folds another aggregation's state (same spec) into `a`, group by group:
 * the merge of two partial aggregates of a partitioned plan (the final
 * half of DataFusion's two-phase aggregate; AVG partials add sum and count). */
static void agg_merge_state(orc_agg* a, const orc_agg* b) {
    for (int64_t gb = 0; gb < b->ngroups; gb++) {
        int64_t g = agg_group(a, b->key_valid[gb], b->keys[gb]);
        for (int32_t j = 0; j < a->n; j++) {
            agg_state* s = &a->st[j];
            const agg_state* t = &b->st[j];
            if (t->cnt[gb] == 0) continue;
            switch (s->func) {
                case ORC_COUNT:
                case ORC_COUNT_STAR: s->cnt[g] += t->cnt[gb]; break;
                case ORC_AVG:
                    s->dval[g] = s->cnt[g] ? s->dval[g] + t->dval[gb] : 0.0 + t->dval[gb];
                    s->cnt[g] += t->cnt[gb];
                    break;
                default: {
                    uint64_t keep = s->cnt[g] + t->cnt[gb];
                    if (s->in_type == ORC_FLOAT64) agg_fold(s, g, 1, 0, t->dval[gb]);
                    else agg_fold(s, g, 0, t->ival[gb], 0.0);
                    s->cnt[g] = keep;
                    break;
                }
            }
        }
    }
}

/* ------------------------------------------------------------------------ */
/* one aggregate, split by key over threads                                 */
/* ------------------------------------------------------------------------ */

typedef struct kp_task {
    const orc_column* cols;
    const orc_leaf* leaves;
    int32_t nleaves;
    int32_t part, nparts;
    orc_agg* agg;
} kp_task;

/* Thread `part` scans every row in order and folds the selected rows whose
 * key hashes to it (the NULL key to part 0): each group still sees its rows
 * in row order, exactly as one sequential update folds them. */
static void* kp_thread(void* p) {
    kp_task* t = (kp_task*)p;
    orc_agg* a = t->agg;
    const orc_column* k = &t->cols[a->group_by];
    for (int64_t row = 0; row < k->length; row++) {
        int v = is_valid(k, row);
        int64_t key = v ? key_at(k, row) : 0;
        int32_t owner = v ? (int32_t)(mix64((uint64_t)key) % (uint64_t)t->nparts) : 0;
        if (owner != t->part) continue;
        if (!row_selected(t->cols, t->leaves, t->nleaves, row)) continue;
        agg_update_row(a, t->cols, agg_group(a, v, key), row);
    }
    return NULL;
}

/* GroupedAggregator::new + update + (finish), cpu/kernels.rs:693-772, for
 * one batch, with the groups split over `threads` by a hash of the key.  The
 * partitions hold disjoint groups, so joining them changes no value: the
 * result is bit-identical to a single-threaded update (a faster checker for
 * large inputs, not another semantics). */
int32_t orc_aggregate_parallel(const orc_column* cols, int32_t ncols, const orc_agg_spec* spec,
                               const orc_leaf* leaves, int32_t nleaves, int32_t threads,
                               orc_agg** out) {
    int rc = leaf_types_ok(cols, ncols, leaves, nleaves);
    if (rc != ORC_OK) return rc;
    if (threads < 1) threads = 1;
    if (threads > 256) threads = 256;
    kp_task tasks[256];
    pthread_t tids[256];
    for (int32_t t = 0; t < threads; t++) {
        tasks[t].cols = cols;
        tasks[t].leaves = leaves;
        tasks[t].nleaves = nleaves;
        tasks[t].part = t;
        tasks[t].nparts = threads;
        rc = orc_agg_new(cols, ncols, spec, &tasks[t].agg);
        if (rc != ORC_OK) {
            for (int32_t u = 0; u < t; u++) orc_agg_free(tasks[u].agg);
            return rc;
        }
    }
    if (threads == 1) kp_thread(&tasks[0]);
    else {
        for (int32_t t = 0; t < threads; t++) pthread_create(&tids[t], NULL, kp_thread, &tasks[t]);
        for (int32_t t = 0; t < threads; t++) pthread_join(tids[t], NULL);
    }
    for (int32_t t = 1; t < threads; t++) {
        agg_merge_state(tasks[0].agg, tasks[t].agg);
        orc_agg_free(tasks[t].agg);
    }
    *out = tasks[0].agg;
    return ORC_OK;
}

/* ------------------------------------------------------------------------ */
/* join + filter + aggregate                                                */
/* ------------------------------------------------------------------------ */

typedef struct ja_task {
    const orc_column* probe;
    const orc_column* build;
    const orc_leaf* leaves;
    int32_t nleaves;
    const orc_join_agg_query* q;
    const orc_join_table* table;
    int64_t lo, hi;
    orc_agg* agg;
} ja_task;

static void ja_run(ja_task* t) {
    const orc_join_agg_query* q = t->q;
    const orc_column* pk = &t->probe[q->probe_key];
    const orc_column* gk = q->group_side == 0 ? &t->probe[q->group_column] : &t->build[q->group_column];
    orc_agg* a = t->agg;
    for (int64_t i = t->lo; i < t->hi; i++) {
        if (!row_selected(t->probe, t->leaves, t->nleaves, i)) continue;
        if (!is_valid(pk, i)) continue;
        uint32_t s, c;
        if (!join_run(t->table, key_at(pk, i), &s, &c)) continue;
        for (uint32_t m = 0; m < c; m++) {
            int64_t b = t->table->rows[s + m];
            int64_t grow = q->group_side == 0 ? i : b;
            int v = is_valid(gk, grow);
            int64_t g = agg_group(a, v, v ? key_at(gk, grow) : 0);
            for (int32_t j = 0; j < a->n; j++) {
                agg_state* st = &a->st[j];
                if (st->func == ORC_COUNT_STAR) {
                    st->cnt[g]++;
                    continue;
                }
                const orc_column* col = q->sides[j] == 0 ? &t->probe[q->columns[j]] : &t->build[q->columns[j]];
                int64_t r = q->sides[j] == 0 ? i : b;
                if (!is_valid(col, r)) continue;
                if (st->func == ORC_COUNT) {
                    st->cnt[g]++;
                    continue;
                }
                if (col->type == ORC_FLOAT64) agg_fold(st, g, 1, 0, get_f64(col, r));
                else if (col->type == ORC_INT64) agg_fold(st, g, 0, get_i64(col, r), 0.0);
                else agg_fold(st, g, 0, get_i32(col, r), 0.0);
            }
        }
    }
}

static void* ja_thread(void* p) {
    ja_task* t = (ja_task*)p;
    ja_run(t);
    return NULL;
}

static int32_t ja_agg_new(const orc_column* probe, const orc_column* build,
                          const orc_join_agg_query* q, orc_agg** out) {
    /* A spec over a virtual schema: column 0 = group key, 1 + j = input j. */
    orc_column cols[1 + ORC_MAX_AGGREGATES];
    orc_agg_spec spec;
    memset(&spec, 0, sizeof spec);
    cols[0] = q->group_side == 0 ? probe[q->group_column] : build[q->group_column];
    spec.group_by = 0;
    spec.naggregates = q->naggregates;
    for (int32_t j = 0; j < q->naggregates; j++) {
        spec.funcs[j] = q->funcs[j];
        spec.columns[j] = 1 + j;
        cols[1 + j] = q->funcs[j] == ORC_COUNT_STAR ? cols[0]
                      : (q->sides[j] == 0 ? probe[q->columns[j]] : build[q->columns[j]]);
    }
    return orc_agg_new(cols, 1 + q->naggregates, &spec, out);
}

/* The config-shaped query `probe JOIN build ON key WHERE <leaves on probe>
 * GROUP BY <col> <aggs>` as the reference's CPU path runs it: JoinTable
 * (cpu/kernels.rs:199) once, JoinMatches order (cpu/kernels.rs:303-342),
 * GroupedAggregator folds (cpu/kernels.rs:679-811).  threads > 1 splits the
 * probe rows into contiguous partitions, aggregates each alone and merges
 * the partials in partition order — DataFusion's partitioned plan; float
 * sums then round differently than one pass (within 1e-12 relative). */
int32_t orc_join_aggregate(const orc_column* probe, int32_t nprobe_cols, const orc_column* build,
                           int32_t nbuild_cols, const orc_leaf* leaves, int32_t nleaves,
                           const orc_join_agg_query* q, int32_t threads, orc_agg** out) {
    int rc = leaf_types_ok(probe, nprobe_cols, leaves, nleaves);
    if (rc != ORC_OK) return rc;
    if (q->probe_key < 0 || q->probe_key >= nprobe_cols || q->build_key < 0 ||
        q->build_key >= nbuild_cols)
        return ORC_ERR_PLAN;
    orc_join_table* table;
    rc = orc_join_build(&build[q->build_key], &table);
    if (rc != ORC_OK) return rc;
    int64_t n = probe[q->probe_key].length;
    if (threads < 1) threads = 1;
    if (threads > 256) threads = 256;
    ja_task tasks[256];
    pthread_t tids[256];
    for (int32_t t = 0; t < threads; t++) {
        tasks[t].probe = probe;
        tasks[t].build = build;
        tasks[t].leaves = leaves;
        tasks[t].nleaves = nleaves;
        tasks[t].q = q;
        tasks[t].table = table;
        tasks[t].lo = n * t / threads;
        tasks[t].hi = n * (t + 1) / threads;
        rc = ja_agg_new(probe, build, q, &tasks[t].agg);
        if (rc != ORC_OK) {
            for (int32_t u = 0; u < t; u++) orc_agg_free(tasks[u].agg);
            orc_join_free(table);
            return rc;
        }
    }
    if (threads == 1) ja_run(&tasks[0]);
    else {
        for (int32_t t = 0; t < threads; t++) pthread_create(&tids[t], NULL, ja_thread, &tasks[t]);
        for (int32_t t = 0; t < threads; t++) pthread_join(tids[t], NULL);
    }
    for (int32_t t = 1; t < threads; t++) {
        agg_merge_state(tasks[0].agg, tasks[t].agg);
        orc_agg_free(tasks[t].agg);
    }
    orc_join_free(table);
    *out = tasks[0].agg;
    return ORC_OK;
}

/* ------------------------------------------------------------------------ */
/* vectors                                                                  */
/* ------------------------------------------------------------------------ */

/* vector_distance, cpu/kernels.rs:841-906: NULL vector → NULL distance. */
int32_t orc_vector_distance(const orc_column* vec, const float* query, int32_t metric, float* out,
                            uint8_t* out_valid) {
    if (vec->type != ORC_VECTOR_F32) return ORC_ERR_UNSUPPORTED;
    int64_t dim = vec->dim;
    const float* v = (const float*)vec->values;
    for (int64_t r = 0; r < vec->length; r++) {
        if (!is_valid(vec, r)) {
            out[r] = 0.0f;
            out_valid[r] = 0;
            continue;
        }
        out[r] = metric == ORC_L2 ? orc_l2(v + r * dim, query, dim) : orc_cosine(v + r * dim, query, dim);
        out_valid[r] = 1;
    }
    return ORC_OK;
}

/* Order of ORDER BY distance, id: Arrow sorts floats in totalOrder (NaN
 * greatest); ties by row id. */
static inline int dist_less(float da, int64_t ia, float db, int64_t ib) {
    int32_t ka = (int32_t)f32_bits(da), kb = (int32_t)f32_bits(db);
    ka ^= (int32_t)(((uint32_t)(ka >> 31)) >> 1);
    kb ^= (int32_t)(((uint32_t)(kb >> 31)) >> 1);
    if (ka != kb) return ka < kb;
    return ia < ib;
}

typedef struct topk_task {
    const orc_column* cols;
    int32_t vec_column;
    const orc_leaf* leaves;
    int32_t nleaves;
    const uint8_t* pass;
    const float* queries;
    int32_t q0, q1, k, metric;
    int64_t* ids;
    float* dist;
} topk_task;

static void topk_run(topk_task* t) {
    const orc_column* vec = &t->cols[t->vec_column];
    int64_t dim = vec->dim, n = vec->length;
    const float* v = (const float*)vec->values;
    int32_t k = t->k;
    float* hd = (float*)malloc((size_t)(k + 1) * 4);
    int64_t* hi = (int64_t*)malloc((size_t)(k + 1) * 8);
    for (int32_t qi = t->q0; qi < t->q1; qi++) {
        const float* q = t->queries + (int64_t)qi * dim;
        int32_t m = 0; /* max-heap on (dist, id) of the best k */
        for (int64_t r = 0; r < n; r++) {
            if (!t->pass[r]) continue;
            float d = t->metric == ORC_L2 ? orc_l2(v + r * dim, q, dim) : orc_cosine(v + r * dim, q, dim);
            if (m < k) {
                int32_t c = m++;
                hd[c] = d;
                hi[c] = r;
                while (c > 0) {
                    int32_t p = (c - 1) / 2;
                    if (!dist_less(hd[p], hi[p], hd[c], hi[c])) break;
                    float td = hd[p]; hd[p] = hd[c]; hd[c] = td;
                    int64_t ti = hi[p]; hi[p] = hi[c]; hi[c] = ti;
                    c = p;
                }
            } else if (k > 0 && dist_less(d, r, hd[0], hi[0])) {
                hd[0] = d;
                hi[0] = r;
                int32_t c = 0;
                for (;;) {
                    int32_t l = 2 * c + 1, rr = l + 1, big = c;
                    if (l < m && dist_less(hd[big], hi[big], hd[l], hi[l])) big = l;
                    if (rr < m && dist_less(hd[big], hi[big], hd[rr], hi[rr])) big = rr;
                    if (big == c) break;
                    float td = hd[big]; hd[big] = hd[c]; hd[c] = td;
                    int64_t ti = hi[big]; hi[big] = hi[c]; hi[c] = ti;
                    c = big;
                }
            }
        }
        /* heap → ascending */
        for (int32_t a = 1; a < m; a++) {
            float d = hd[a];
            int64_t id = hi[a];
            int32_t b = a - 1;
            while (b >= 0 && dist_less(d, id, hd[b], hi[b])) {
                hd[b + 1] = hd[b];
                hi[b + 1] = hi[b];
                b--;
            }
            hd[b + 1] = d;
            hi[b + 1] = id;
        }
        for (int32_t j = 0; j < k; j++) {
            t->ids[(int64_t)qi * k + j] = j < m ? hi[j] : -1;
            t->dist[(int64_t)qi * k + j] = j < m ? hd[j] : NAN;
        }
    }
    free(hd);
    free(hi);
}

static void* topk_thread(void* p) {
    topk_run((topk_task*)p);
    return NULL;
}

/* ORDER BY l2|cosine(vec, q) LIMIT k over the rows a WHERE keeps: the
 * reference runs vector_distance (cpu/kernels.rs:841) then DataFusion's
 * SortExec(fetch=k); rows with a NULL vector have a NULL distance, which
 * sorts last, and are left out here. */
int32_t orc_vector_topk(const orc_column* cols, int32_t ncols, int32_t vec_column,
                        const orc_leaf* leaves, int32_t nleaves, const float* queries,
                        int32_t nqueries, int32_t k, int32_t metric, int32_t threads,
                        int64_t* out_ids, float* out_dist) {
    if (vec_column < 0 || vec_column >= ncols) return ORC_ERR_PLAN;
    if (cols[vec_column].type != ORC_VECTOR_F32) return ORC_ERR_UNSUPPORTED;
    int rc = leaf_types_ok(cols, ncols, leaves, nleaves);
    if (rc != ORC_OK) return rc;
    int64_t n = cols[vec_column].length;
    uint8_t* pass = (uint8_t*)malloc((size_t)n + 1);
    for (int64_t r = 0; r < n; r++)
        pass[r] = (uint8_t)(is_valid(&cols[vec_column], r) && row_selected(cols, leaves, nleaves, r));
    if (threads < 1) threads = 1;
    if (threads > 256) threads = 256;
    if (threads > nqueries) threads = nqueries > 0 ? nqueries : 1;
    topk_task tasks[256];
    pthread_t tids[256];
    for (int32_t t = 0; t < threads; t++) {
        topk_task* x = &tasks[t];
        x->cols = cols;
        x->vec_column = vec_column;
        x->leaves = leaves;
        x->nleaves = nleaves;
        x->pass = pass;
        x->queries = queries;
        x->q0 = (int32_t)((int64_t)nqueries * t / threads);
        x->q1 = (int32_t)((int64_t)nqueries * (t + 1) / threads);
        x->k = k;
        x->metric = metric;
        x->ids = out_ids;
        x->dist = out_dist;
    }
    if (threads == 1) topk_run(&tasks[0]);
    else {
        for (int32_t t = 0; t < threads; t++) pthread_create(&tids[t], NULL, topk_thread, &tasks[t]);
        for (int32_t t = 0; t < threads; t++) pthread_join(tids[t], NULL);
    }
    free(pass);
    return ORC_OK;
}
