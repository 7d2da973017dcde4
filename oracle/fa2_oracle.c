/*
 * ORACLE — test infrastructure only.
 *
 * A CPU, FP64 restatement of graph-core's ForceAtlas2 tick (the reference's
 * `layout.forceatlas2` / `layout.forceatlas2.barnes_hut` arms) that the CUDA
 * engine is checked against. Only tests/, __graft_entry__.smoke() and bench.py's
 * CPU-baseline leg load it. It is never linked into the product library.
 *
 * Parity pins (checked by tests/test_oracle.py):
 *   - crates/graph-cli/tests/fixtures/fa2-nx-reference.jsonl (networkx 3.6 at 2
 *     iterations over the gate model, seeds 0..63) within the reference's own
 *     ceiling of 1e-7 of the layout extent (graph-cli/src/oracle_python/fa2.rs:72-78);
 *   - live networkx 3.6.1 `forceatlas2_layout` for the options graph-core does not
 *     implement (linlog, distributed_action, strong_gravity, weights, dim 3);
 *   - theta = 0 tree == dense (state/barnes_hut/tests.rs:60-70), the theta = 0.8
 *     error bound (barnes_hut/tests.rs:73-88), the gravity association bit-pin
 *     (state/tests.rs:27-62) and the coincident-pair jiggle (state/tests.rs:69-94).
 *
 * Every function cites the reference file:line it restates. Paths are relative to
 * crates/graph-core/src/ unless they say otherwise.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define MAXD 3
#define DBL_MIN_POS 2.2250738585072014e-308 /* f64::MIN_POSITIVE */

/* ---------------------------------------------------------------- rng ---- */

/* Mulberry32, synthetic.rs:37-50: integer steps, then / 2^32. */
typedef struct { uint32_t s; } orc_mb32;

static double mb_next(orc_mb32 *r) {
    r->s += 0x6D2B79F5u;
    uint32_t a = r->s;
    uint32_t t = (a ^ (a >> 15)) * (1u | a);
    t = (t + ((t ^ (t >> 7)) * (61u | t))) ^ t;
    return (double)(t ^ (t >> 14)) / 4294967296.0;
}

/* Mulberry32::pick, synthetic.rs:52-61: floor(next * len). */
static uint32_t mb_pick(orc_mb32 *r, uint32_t len) {
    return (uint32_t)floor(mb_next(r) * (double)len);
}

/* state.rs:272-283: dim draws per node, ascending axis. Row-major n x dim. */
void orc_initial_positions(uint32_t n, uint32_t seed, int dim, double *out) {
    orc_mb32 r = {seed};
    for (uint32_t i = 0; i < n; i++)
        for (int a = 0; a < dim; a++) out[(size_t)i * dim + a] = mb_next(&r);
}

/* rng.rs:27-34, MurmurHash3 fmix64. */
static uint64_t fmix64(uint64_t k) {
    k ^= k >> 33;
    k *= 0xff51afd7ed558ccdULL;
    k ^= k >> 33;
    k *= 0xc4ceb9fe1a85ec53ULL;
    k ^= k >> 33;
    return k;
}

/* rng.rs:39-44 (fold) and 61-84 (jiggle, jiggle_of). */
double orc_jiggle(uint32_t seed, uint32_t tick, uint32_t pass, uint32_t i, uint32_t j) {
    uint32_t lo = i <= j ? i : j, hi = i <= j ? j : i;
    uint64_t a = fmix64((uint64_t)seed ^ ((uint64_t)tick << 32));
    uint64_t b = fmix64(a ^ ((uint64_t)pass << 32) ^ (uint64_t)lo);
    uint64_t w = fmix64(b ^ ((uint64_t)hi << 32) ^ a) >> 11;
    if (w == (1ULL << 52)) w = (1ULL << 52) + 1;
    double u = (double)w * (1.0 / (double)(1ULL << 53));
    return (u - 0.5) * 1e-6;
}

/* ------------------------------------------------------ gate model ------ */

/* synthetic_records + synthetic_edges, synthetic.rs:92-170: the draws the
 * node records consume (icon roll, table pick), then preferential attachment and
 * the 5% note-link extras. A self-edge draws no strength. Writes at most `cap`
 * edges; returns how many the model has. */
int64_t orc_gate_edges(uint32_t count, uint32_t *src, uint32_t *dst, double *strength,
                       int64_t cap) {
    orc_mb32 r = {0x051042u};
    for (uint32_t i = 0; i < count; i++) {
        double roll = mb_next(&r);
        if (roll < 0.6)
            (void)mb_pick(&r, 12);
        else if (roll < 0.8)
            (void)mb_pick(&r, 4);
    }
    int64_t m = 0;
#define PUSH(A, B)                                                     \
    do {                                                               \
        uint32_t a_ = (A), b_ = (B);                                   \
        if (a_ != b_) {                                                \
            double s_ = 0.4 + mb_next(&r) * 0.4;                       \
            if (m < cap) { src[m] = a_; dst[m] = b_; strength[m] = s_; } \
            m++;                                                       \
        }                                                              \
    } while (0)
    for (uint32_t i = 1; i < count; i++) {
        double x = mb_next(&r), y = mb_next(&r);
        PUSH(i, (uint32_t)floor(x * y * (double)i));
        if (mb_next(&r) < 0.5) {
            x = mb_next(&r);
            y = mb_next(&r);
            PUSH(i, (uint32_t)floor(x * y * (double)i));
        }
    }
    uint32_t extras = (uint32_t)floor((double)count * 0.05);
    for (uint32_t e = 0; e < extras; e++) {
        uint32_t a = mb_pick(&r, count), b = mb_pick(&r, count);
        PUSH(a, b);
    }
#undef PUSH
    return m;
}

/* ------------------------------------------------------ simple graph ---- */

/* layout/force/mod.rs:101-120: drop self-loops, keep the first raw edge of each
 * unordered pair (ascending edge index), lo < hi. Uses an open-addressing table
 * keyed on the pair; output order is first-arrival order, as IndexMap keeps it.
 * Returns the simple edge count. */
int64_t orc_simple_graph(uint32_t n, int64_t m, const uint32_t *src, const uint32_t *dst,
                         const double *w, uint32_t *lo, uint32_t *hi, double *wout) {
    (void)n;
    uint64_t cap = 16;
    while (cap < (uint64_t)m * 2 + 16) cap <<= 1;
    uint64_t *table = (uint64_t *)malloc(cap * sizeof(uint64_t));
    for (uint64_t i = 0; i < cap; i++) table[i] = UINT64_MAX;
    int64_t k = 0;
    for (int64_t e = 0; e < m; e++) {
        uint32_t a = src[e], b = dst[e];
        if (a == b) continue;
        uint32_t l = a < b ? a : b, h = a < b ? b : a;
        uint64_t key = ((uint64_t)l << 32) | h;
        uint64_t slot = fmix64(key) & (cap - 1);
        int seen = 0;
        while (table[slot] != UINT64_MAX) {
            if (table[slot] == key) { seen = 1; break; }
            slot = (slot + 1) & (cap - 1);
        }
        if (seen) continue;
        table[slot] = key;
        lo[k] = l;
        hi[k] = h;
        wout[k] = w ? w[e] : 1.0;
        k++;
    }
    free(table);
    return k;
}

/* ---------------------------------------------------------- params ------ */

/* Fa2Params (state.rs:20-54) plus the options networkx 3.6 publishes and
 * graph-core leaves at their defaults (layout.py:1604-1875). theta < 0 selects the
 * dense O(n^2) repulsion (state.rs:169-183); theta >= 0 the tree walk
 * (barnes_hut.rs:115-184) at that opening angle. depth_cap > 0 stops the tree at
 * that many levels below the root square (points still together there share one
 * leaf), which is the tree a fixed-width Morton key describes. */
typedef struct {
    int64_t max_iter;
    double jitter_tolerance;
    double scaling_ratio;
    double gravity;
    int64_t seed;
    int64_t dim;
    double theta;
    int64_t lin_log;
    int64_t strong_gravity;
    int64_t dissuade_hubs;
    double edge_weight_influence;
    int64_t depth_cap;
    int64_t threads;
} orc_params;

/* ------------------------------------------------------------ tree ------ */

/* quadtree.rs:20-25 Shape, generalised to 2^dim children (octree.rs uses the
 * same algorithm with three bits per slot). */
typedef struct {
    int32_t child[1 << MAXD];
    int32_t head; /* >= 0: leaf, the chain head point; -1: internal */
    int32_t depth;
} tshape;

/* preorder.rs:21-41 Cell. */
typedef struct {
    double b0[MAXD], b1[MAXD];
    uint32_t skip, start, end;
} tcell;

typedef struct {
    double mass, c[MAXD];
} tbody;

typedef struct {
    int dim;
    int depth_cap;
    double r0[MAXD], r1[MAXD];
    int root_set; /* root square initialised by the first cover */
    tshape *shape;
    size_t nshape, capshape;
    int32_t root;
    int32_t *chain_next;
    tcell *cells;
    int32_t *node_id; /* preorder cell -> its arena (shape) index, quadtree.rs node_id */
    size_t ncells, capcells;
    uint32_t *order;
    size_t norder;
    tbody *bodies;
    size_t capbodies;
} ttree;

static void tree_reset(ttree *t, uint32_t n, int dim, int cap) {
    t->dim = dim;
    t->depth_cap = cap;
    t->root_set = 0;
    t->nshape = 0;
    t->root = -1;
    t->ncells = 0;
    t->norder = 0;
    t->chain_next = (int32_t *)realloc(t->chain_next, (size_t)(n ? n : 1) * sizeof(int32_t));
    for (uint32_t i = 0; i < n; i++) t->chain_next[i] = -1;
    t->order = (uint32_t *)realloc(t->order, (size_t)(n ? n : 1) * sizeof(uint32_t));
}

static int32_t tree_push(ttree *t, int32_t head, int32_t depth) {
    if (t->nshape == t->capshape) {
        t->capshape = t->capshape ? t->capshape * 2 : 1024;
        t->shape = (tshape *)realloc(t->shape, t->capshape * sizeof(tshape));
    }
    tshape *s = &t->shape[t->nshape];
    for (int c = 0; c < (1 << MAXD); c++) s->child[c] = -1;
    s->head = head;
    s->depth = depth;
    return (int32_t)(t->nshape++);
}

/* quadtree.rs:157-195 cover (d3 cover.js), generalised per axis: the first point
 * sets [floor(x), floor(x)+1); later points double the square away from the side
 * they fall on until it holds them. */
static void tree_cover(ttree *t, const double *x) {
    int d = t->dim;
    if (!t->root_set) {
        for (int a = 0; a < d; a++) {
            t->r1[a] = floor(x[a]) + 1.0;
            t->r0[a] = t->r1[a] - 1.0;
        }
        t->root_set = 1;
        return;
    }
    double z = (t->r1[0] - t->r0[0] != 0.0) ? t->r1[0] - t->r0[0] : 1.0;
    for (;;) {
        int inside = 1;
        for (int a = 0; a < d; a++)
            if (t->r0[a] > x[a] || x[a] >= t->r1[a]) inside = 0;
        if (inside) return;
        z *= 2.0;
        for (int a = 0; a < d; a++) {
            if (x[a] < t->r0[a])
                t->r0[a] = t->r1[a] - z;
            else
                t->r1[a] = t->r0[a] + z;
        }
        if (!(isfinite(z) && isfinite(t->r1[0] - t->r0[0]))) return;
    }
}

/* bounds.rs:34-50 narrow: the slot whose bit a is (x[a] >= mid[a]). */
static int narrow(int d, double *b0, double *b1, const double *x) {
    int slot = 0;
    for (int a = 0; a < d; a++) {
        double m = (b0[a] + b1[a]) / 2.0;
        if (x[a] >= m) {
            b0[a] = m;
            slot |= 1 << a;
        } else {
            b1[a] = m;
        }
    }
    return slot;
}

static void tree_attach(ttree *t, int32_t parent, int slot, int32_t child) {
    if (parent >= 0)
        t->shape[parent].child[slot] = child;
    else
        t->root = child;
}

static void tree_chain(ttree *t, uint32_t point, int32_t node) {
    t->chain_next[point] = t->shape[node].head;
    t->shape[node].head = (int32_t)point;
}

/* build.rs:26-96 add + insert_leaf. With depth_cap > 0 a split that would go
 * below depth_cap chains instead, the same way the reference chains two points
 * its f64 midpoints can no longer separate (build.rs:81-85). */
static void tree_add(ttree *t, const double *pos, uint32_t point) {
    int d = t->dim;
    const double *x = pos + (size_t)point * MAXD;
    for (int a = 0; a < d; a++)
        if (!isfinite(x[a])) return;
    if (t->root < 0) {
        t->root = tree_push(t, (int32_t)point, 0);
        return;
    }
    double b0[MAXD], b1[MAXD];
    memcpy(b0, t->r0, sizeof b0);
    memcpy(b1, t->r1, sizeof b1);
    int32_t node = t->root, parent = -1;
    int pslot = 0;
    for (;;) {
        if (t->shape[node].head < 0) {
            int slot = narrow(d, b0, b1, x);
            int32_t c = t->shape[node].child[slot];
            if (c >= 0) {
                parent = node;
                pslot = slot;
                node = c;
                continue;
            }
            int32_t leaf = tree_push(t, (int32_t)point, t->shape[node].depth + 1);
            t->shape[node].child[slot] = leaf;
            return;
        }
        break;
    }
    /* insert_leaf */
    const double *xp = pos + (size_t)t->shape[node].head * MAXD;
    int same = 1;
    for (int a = 0; a < d; a++)
        if (x[a] != xp[a]) same = 0;
    if (same) {
        tree_chain(t, point, node);
        return;
    }
    int32_t at = parent;
    int slot = pslot;
    int32_t depth = t->shape[node].depth;
    for (;;) {
        double before = b1[0] - b0[0];
        if (t->depth_cap > 0 && depth >= t->depth_cap) {
            tree_attach(t, at, slot, node);
            tree_chain(t, point, node);
            return;
        }
        double mid[MAXD];
        for (int a = 0; a < d; a++) mid[a] = (b0[a] + b1[a]) / 2.0;
        int i = narrow(d, b0, b1, x);
        int j = 0;
        for (int a = 0; a < d; a++)
            if (xp[a] >= mid[a]) j |= 1 << a;
        double after = b1[0] - b0[0];
        if (!(after < before)) {
            tree_attach(t, at, slot, node);
            tree_chain(t, point, node);
            return;
        }
        int32_t internal = tree_push(t, -1, depth);
        tree_attach(t, at, slot, internal);
        depth++;
        t->shape[node].depth = depth;
        if (i != j) {
            t->shape[internal].child[j] = node;
            int32_t leaf = tree_push(t, (int32_t)point, depth);
            t->shape[internal].child[i] = leaf;
            return;
        }
        at = internal;
        slot = i;
    }
}

static void cell_push(ttree *t, const double *b0, const double *b1, uint32_t start, int32_t node) {
    if (t->ncells == t->capcells) {
        t->capcells = t->capcells ? t->capcells * 2 : 1024;
        t->cells = (tcell *)realloc(t->cells, t->capcells * sizeof(tcell));
        t->node_id = (int32_t *)realloc(t->node_id, t->capcells * sizeof(int32_t));
    }
    t->node_id[t->ncells] = node;
    tcell *c = &t->cells[t->ncells++];
    memcpy(c->b0, b0, sizeof c->b0);
    memcpy(c->b1, b1, sizeof c->b1);
    c->start = start;
    c->skip = 0;
    c->end = 0;
}

/* preorder.rs:56-114 flatten/open: cells in preorder, children in slot order,
 * each cell's bounds from bounds.rs:84-108 quadrant; then the non-finite points. */
typedef struct {
    int32_t node;
    int close; /* 1: close cell `node` */
    double b0[MAXD], b1[MAXD];
} visit;

static void tree_flatten(ttree *t, const double *pos, uint32_t n) {
    int d = t->dim;
    size_t cap = 1024, top = 0;
    visit *stack = (visit *)malloc(cap * sizeof(visit));
    if (t->root >= 0) {
        stack[top].node = t->root;
        stack[top].close = 0;
        memcpy(stack[top].b0, t->r0, sizeof t->r0);
        memcpy(stack[top].b1, t->r1, sizeof t->r1);
        top++;
    }
    while (top) {
        visit v = stack[--top];
        if (v.close) {
            t->cells[v.node].skip = (uint32_t)t->ncells;
            t->cells[v.node].end = (uint32_t)t->norder;
            continue;
        }
        uint32_t k = (uint32_t)t->ncells;
        uint32_t start = (uint32_t)t->norder;
        cell_push(t, v.b0, v.b1, start, v.node);
        tshape *s = &t->shape[v.node];
        if (s->head >= 0) {
            for (int32_t p = s->head; p >= 0; p = t->chain_next[p]) t->order[t->norder++] = (uint32_t)p;
            t->cells[k].end = (uint32_t)t->norder;
            t->cells[k].skip = k + 1;
            continue;
        }
        if (top + (1 << MAXD) + 2 > cap) {
            cap *= 2;
            stack = (visit *)realloc(stack, cap * sizeof(visit));
        }
        stack[top].node = (int32_t)k;
        stack[top].close = 1;
        top++;
        for (int slot = (1 << d) - 1; slot >= 0; slot--) {
            int32_t c = s->child[slot];
            if (c < 0) continue;
            visit *w = &stack[top++];
            w->node = c;
            w->close = 0;
            for (int a = 0; a < d; a++) {
                double m = (v.b0[a] + v.b1[a]) / 2.0;
                if (slot & (1 << a)) {
                    w->b0[a] = m;
                    w->b1[a] = v.b1[a];
                } else {
                    w->b0[a] = v.b0[a];
                    w->b1[a] = m;
                }
            }
            for (int a = d; a < MAXD; a++) w->b0[a] = w->b1[a] = 0.0;
        }
    }
    free(stack);
    for (uint32_t i = 0; i < n; i++) {
        const double *x = pos + (size_t)i * MAXD;
        int ok = 1;
        for (int a = 0; a < d; a++)
            if (!isfinite(x[a])) ok = 0;
        if (!ok) t->order[t->norder++] = i;
    }
}

/* quadtree.rs:116-140 build: extent of the finite points (quadtree.rs:46-53),
 * cover both corners, insert ascending, flatten. */
static void tree_build(ttree *t, const double *pos, uint32_t n, int dim, int cap) {
    tree_reset(t, n, dim, cap);
    double lo[MAXD], hi[MAXD];
    int any = 0;
    for (uint32_t i = 0; i < n; i++) {
        const double *x = pos + (size_t)i * MAXD;
        int ok = 1;
        for (int a = 0; a < dim; a++)
            if (!isfinite(x[a])) ok = 0;
        if (!ok) continue;
        for (int a = 0; a < dim; a++) {
            if (!any || x[a] < lo[a]) lo[a] = x[a];
            if (!any || x[a] > hi[a]) hi[a] = x[a];
        }
        any = 1;
    }
    if (any) {
        tree_cover(t, lo);
        tree_cover(t, hi);
        for (uint32_t i = 0; i < n; i++) tree_add(t, pos, i);
    }
    tree_flatten(t, pos, n);
}

/* ----------------------------------------------------------- state ------ */

typedef struct {
    orc_params P;
    uint32_t n;
    int64_t m;
    int dim;
    uint32_t *lo, *hi;
    double *w; /* effective attraction weight per simple edge, w^influence */
    double *p, *u, *mass;
    uint32_t iter_no;
    double swing, traction, speed, speed_efficiency;
    ttree tree;
    uint64_t far_count, pair_count;
} orc_fa2;

static double norm2(const double *v, int dim) {
    double s = 0.0;
    for (int a = 0; a < dim; a++) s += v[a] * v[a];
    return s;
}

/* state.rs:83-102 Fa2State::new over an already-simple edge list: mass =
 * degree + 1, positions from pos0 (row-major n x dim) or Mulberry32(seed). */
orc_fa2 *orc_fa2_new(uint32_t n, int64_t m, const uint32_t *lo, const uint32_t *hi,
                     const double *w, const orc_params *params, const double *pos0) {
    orc_fa2 *s = (orc_fa2 *)calloc(1, sizeof(orc_fa2));
    s->P = *params;
    s->n = n;
    s->m = m;
    s->dim = (int)params->dim;
    size_t nn = n ? n : 1, mm = m ? (size_t)m : 1;
    s->lo = (uint32_t *)malloc(mm * sizeof(uint32_t));
    s->hi = (uint32_t *)malloc(mm * sizeof(uint32_t));
    s->w = (double *)malloc(mm * sizeof(double));
    s->p = (double *)calloc(nn * MAXD, sizeof(double));
    s->u = (double *)calloc(nn * MAXD, sizeof(double));
    s->mass = (double *)calloc(nn, sizeof(double));
    for (int64_t e = 0; e < m; e++) {
        s->lo[e] = lo[e];
        s->hi[e] = hi[e];
        double we = w ? w[e] : 1.0;
        s->w[e] = params->edge_weight_influence == 0.0 ? 1.0
                  : params->edge_weight_influence == 1.0 ? we
                                                         : pow(we, params->edge_weight_influence);
        s->mass[lo[e]] += 1.0;
        s->mass[hi[e]] += 1.0;
    }
    for (uint32_t i = 0; i < n; i++) s->mass[i] += 1.0;
    if (pos0) {
        for (uint32_t i = 0; i < n; i++)
            for (int a = 0; a < s->dim; a++) s->p[(size_t)i * MAXD + a] = pos0[(size_t)i * s->dim + a];
    } else {
        orc_mb32 r = {(uint32_t)params->seed};
        for (uint32_t i = 0; i < n; i++)
            for (int a = 0; a < s->dim; a++) s->p[(size_t)i * MAXD + a] = mb_next(&r);
    }
    s->swing = s->traction = s->speed = s->speed_efficiency = 1.0;
    return s;
}

void orc_fa2_free(orc_fa2 *s) {
    if (!s) return;
    free(s->lo);
    free(s->hi);
    free(s->w);
    free(s->p);
    free(s->u);
    free(s->mass);
    free(s->tree.shape);
    free(s->tree.chain_next);
    free(s->tree.cells);
    free(s->tree.node_id);
    free(s->tree.order);
    free(s->tree.bodies);
    free(s);
}

/* state.rs:152-162 attraction, with networkx's linlog (layout.py:1806-1811),
 * weights (`A = to_numpy_array(G, weight)`) and distributed_action (1815-1816). */
static void attraction(orc_fa2 *s) {
    int d = s->dim;
    for (int64_t e = 0; e < s->m; e++) {
        double *pl = s->p + (size_t)s->lo[e] * MAXD, *ph = s->p + (size_t)s->hi[e] * MAXD;
        double *ul = s->u + (size_t)s->lo[e] * MAXD, *uh = s->u + (size_t)s->hi[e] * MAXD;
        double diff[MAXD];
        for (int a = 0; a < d; a++) diff[a] = ph[a] - pl[a];
        double c = s->w[e];
        if (s->P.lin_log) {
            double dist = sqrt(norm2(diff, d));
            c *= dist > 0.0 ? log(1.0 + dist) / dist : 0.0;
        }
        if (c == 1.0) {
            for (int a = 0; a < d; a++) {
                ul[a] += diff[a];
                uh[a] -= diff[a];
            }
        } else {
            for (int a = 0; a < d; a++) {
                ul[a] += diff[a] * c;
                uh[a] -= diff[a] * c;
            }
        }
    }
    if (s->P.dissuade_hubs)
        for (uint32_t i = 0; i < s->n; i++)
            for (int a = 0; a < d; a++) s->u[(size_t)i * MAXD + a] /= s->mass[i];
}

/* state.rs:185-203 repel_delta: p_i - p_j, or the counter-hash jiggle on every
 * axis when every live axis is exactly zero. */
static void repel_delta(const orc_fa2 *s, uint32_t i, uint32_t j, double *dlt) {
    int d = s->dim, zero = 1;
    for (int a = 0; a < d; a++) {
        dlt[a] = s->p[(size_t)i * MAXD + a] - s->p[(size_t)j * MAXD + a];
        if (dlt[a] != 0.0) zero = 0;
    }
    if (zero)
        for (int a = 0; a < d; a++)
            dlt[a] = orc_jiggle((uint32_t)s->P.seed, s->iter_no, (uint32_t)a, i, j);
}

/* state.rs:169-183: dense repulsion, one unordered pair at a time. */
static void repulsion_dense(orc_fa2 *s) {
    uint32_t n = s->n;
    int d = s->dim;
    double k = s->P.scaling_ratio;
    for (uint32_t i = 0; i < n; i++)
        for (uint32_t j = i + 1; j < n; j++) {
            double dl[MAXD];
            repel_delta(s, i, j, dl);
            double f = s->mass[i] * s->mass[j] / norm2(dl, d) * k;
            for (int a = 0; a < d; a++) {
                s->u[(size_t)i * MAXD + a] += dl[a] * f;
                s->u[(size_t)j * MAXD + a] -= dl[a] * f;
            }
        }
    s->pair_count += (uint64_t)n * (n ? n - 1 : 0);
}

/* barnes_hut.rs:65-110 aggregate / leaf_sum / children_sum. */
static void tree_aggregate(orc_fa2 *s) {
    ttree *t = &s->tree;
    int d = s->dim;
    if (t->capbodies < t->ncells) {
        t->capbodies = t->ncells;
        t->bodies = (tbody *)realloc(t->bodies, t->capbodies * sizeof(tbody));
    }
    for (size_t kk = t->ncells; kk-- > 0;) {
        tcell *c = &t->cells[kk];
        tbody b;
        memset(&b, 0, sizeof b);
        if (c->skip == kk + 1) {
            for (uint32_t q = c->start; q < c->end; q++) {
                uint32_t pt = t->order[q];
                double mm = s->mass[pt];
                b.mass += mm;
                for (int a = 0; a < d; a++) b.c[a] += mm * s->p[(size_t)pt * MAXD + a];
            }
        } else {
            size_t ch = kk + 1;
            while (ch < c->skip) {
                b.mass += t->bodies[ch].mass;
                for (int a = 0; a < d; a++) b.c[a] += t->bodies[ch].c[a];
                ch = t->cells[ch].skip;
            }
        }
        t->bodies[kk] = b;
    }
    for (size_t kk = 0; kk < t->ncells; kk++)
        for (int a = 0; a < d; a++) t->bodies[kk].c[a] = t->bodies[kk].c[a] / t->bodies[kk].mass;
}

/* barnes_hut.rs:163-184 pairs: the exact force on i from the rest of one leaf. */
static void leaf_pairs(const orc_fa2 *s, uint32_t i, uint32_t q0, uint32_t q1, double *f) {
    int d = s->dim;
    double k = s->P.scaling_ratio;
    for (uint32_t q = q0; q < q1; q++) {
        uint32_t j = s->tree.order[q];
        if (j == i) continue;
        double dl[MAXD];
        if (i < j) {
            repel_delta(s, i, j, dl);
        } else {
            repel_delta(s, j, i, dl);
            for (int a = 0; a < d; a++) dl[a] = -dl[a];
        }
        double fac = s->mass[i] * s->mass[j] / norm2(dl, d) * k;
        for (int a = 0; a < d; a++) f[a] += dl[a] * fac;
    }
}

/* barnes_hut.rs:128-159 walk: stackless preorder; a cell that does not hold the
 * node and satisfies w^2 < theta^2 d^2 acts as one body. */
static void tree_walk(const orc_fa2 *s, uint32_t p, double theta2, double *f, uint64_t *nfar,
                      uint64_t *npair) {
    const ttree *t = &s->tree;
    int d = s->dim;
    uint32_t i = t->order[p];
    const double *xi = s->p + (size_t)i * MAXD;
    double mi = s->mass[i], kr = s->P.scaling_ratio;
    for (int a = 0; a < d; a++) f[a] = 0.0;
    size_t k = 0;
    while (k < t->ncells) {
        const tcell *c = &t->cells[k];
        int holds = c->start <= p && p < c->end;
        const tbody *b = &t->bodies[k];
        double dl[MAXD];
        for (int a = 0; a < d; a++) dl[a] = xi[a] - b->c[a];
        double d2 = norm2(dl, d);
        double w = c->b1[0] - c->b0[0];
        if (!holds && d2 > 0.0 && w * w < theta2 * d2) {
            double fac = mi * b->mass / d2 * kr;
            for (int a = 0; a < d; a++) f[a] = f[a] + dl[a] * fac;
            (*nfar)++;
            k = c->skip;
        } else if (c->skip == k + 1) {
            leaf_pairs(s, i, c->start, c->end, f);
            *npair += (c->end - c->start) - (holds ? 1 : 0);
            k++;
        } else {
            k++;
        }
    }
}

/* barnes_hut.rs:115-125 repel_tree. Per-node walks are independent gathers, so
 * the OpenMP arm visits them in parallel with bit-identical output. */
static void repulsion_tree(orc_fa2 *s) {
    int d = s->dim;
    tree_build(&s->tree, s->p, s->n, d, (int)s->P.depth_cap);
    tree_aggregate(s);
    double theta2 = s->P.theta * s->P.theta;
    uint64_t nfar = 0, npair = 0;
    long np = (long)s->tree.norder;
#ifdef _OPENMP
    int threads = s->P.threads > 0 ? (int)s->P.threads : 1;
#pragma omp parallel for schedule(dynamic, 256) num_threads(threads) reduction(+ : nfar, npair)
#endif
    for (long p = 0; p < np; p++) {
        uint32_t i = s->tree.order[p];
        const double *xi = s->p + (size_t)i * MAXD;
        int ok = 1;
        for (int a = 0; a < d; a++)
            if (!isfinite(xi[a])) ok = 0;
        if (!ok) continue;
        double f[MAXD];
        uint64_t lf = 0, lp = 0;
        tree_walk(s, (uint32_t)p, theta2, f, &lf, &lp);
        nfar += lf;
        npair += lp;
        for (int a = 0; a < d; a++) s->u[(size_t)i * MAXD + a] += f[a];
    }
    s->far_count += nfar;
    s->pair_count += npair;
}

/* state.rs:208-218 mean, ascending. */
static void pos_mean(const orc_fa2 *s, double *mean) {
    int d = s->dim;
    for (int a = 0; a < MAXD; a++) mean[a] = 0.0;
    for (uint32_t i = 0; i < s->n; i++)
        for (int a = 0; a < d; a++) mean[a] += s->p[(size_t)i * MAXD + a];
    for (int a = 0; a < d; a++) mean[a] /= (double)s->n;
}

/* state.rs:223-251 gravity (unit vector first: state/tests.rs:27-62), and
 * networkx's strong_gravity (layout.py:1830-1832). */
static void gravity(orc_fa2 *s) {
    uint32_t n = s->n;
    int d = s->dim;
    if (n == 0) return;
    double mean[MAXD];
    pos_mean(s, mean);
    for (uint32_t i = 0; i < n; i++) {
        double c[MAXD];
        for (int a = 0; a < d; a++) c[a] = s->p[(size_t)i * MAXD + a] - mean[a];
        double g = s->P.gravity * s->mass[i];
        double *ui = s->u + (size_t)i * MAXD;
        if (s->P.strong_gravity) {
            for (int a = 0; a < d; a++) ui[a] -= g * c[a];
        } else {
            double norm = sqrt(norm2(c, d));
            for (int a = 0; a < d; a++) {
                double unit = norm > 0.0 ? c[a] / norm : 0.0;
                ui[a] -= g * unit;
            }
        }
    }
}

/* The force accumulator `u` of one tick at the current positions
 * (state.rs:130-137): attraction, repulsion, gravity. terms: bit 0 attraction,
 * bit 1 repulsion, bit 2 gravity. */
void orc_fa2_accumulate(orc_fa2 *s, int terms) {
    memset(s->u, 0, (size_t)(s->n ? s->n : 1) * MAXD * sizeof(double));
    if (terms & 1) attraction(s);
    if (terms & 2) {
        if (s->P.theta < 0.0)
            repulsion_dense(s);
        else
            repulsion_tree(s);
    }
    if (terms & 4) gravity(s);
}

/* schedule.rs:16-30 swing_and_traction. */
static void swing_traction(const orc_fa2 *s, double *sw, double *tr) {
    int d = s->dim;
    double swing = 0.0, traction = 0.0;
    for (uint32_t i = 0; i < s->n; i++) {
        double back[MAXD], fwd[MAXD];
        for (int a = 0; a < d; a++) {
            back[a] = s->p[(size_t)i * MAXD + a] - s->u[(size_t)i * MAXD + a];
            fwd[a] = s->p[(size_t)i * MAXD + a] + s->u[(size_t)i * MAXD + a];
        }
        swing += s->mass[i] * sqrt(norm2(back, d));
        traction += 0.5 * s->mass[i] * sqrt(norm2(fwd, d));
    }
    *sw = swing;
    *tr = traction;
}

/* schedule.rs:33-60 estimate_factor (networkx's helper). */
static void estimate_factor(orc_fa2 *s, double swing, double traction) {
    double n = (double)s->n, jt = s->P.jitter_tolerance;
    double opt_jitter = 0.05 * sqrt(n);
    double min_jitter = sqrt(opt_jitter);
    double min_speed_efficiency = 0.05;
    double other = fmin(10.0, opt_jitter * traction / (n * n));
    double jitter = jt * fmax(min_jitter, other);
    if (swing / traction > 2.0) {
        if (s->speed_efficiency > min_speed_efficiency) s->speed_efficiency *= 0.5;
        jitter = fmax(jitter, jt);
    }
    double target = swing == 0.0 ? INFINITY : jitter * s->speed_efficiency * traction / swing;
    if (swing > jitter * traction) {
        if (s->speed_efficiency > min_speed_efficiency) s->speed_efficiency *= 0.7;
    } else if (s->speed < 1000.0) {
        s->speed_efficiency *= 1.3;
    }
    s->speed += fmin(target - s->speed, 0.5 * s->speed);
}

/* schedule.rs:62-77 apply_update; returns the summed |step|. */
static double apply_update(orc_fa2 *s) {
    int d = s->dim;
    double moved = 0.0;
    for (uint32_t i = 0; i < s->n; i++) {
        double *ui = s->u + (size_t)i * MAXD, *pi = s->p + (size_t)i * MAXD;
        double norm = sqrt(norm2(ui, d));
        double factor = s->speed / (1.0 + sqrt(s->speed * s->mass[i] * norm));
        double step = 0.0;
        for (int a = 0; a < d; a++) {
            double dd = ui[a] * factor;
            pi[a] += dd;
            step += fabs(dd);
        }
        moved += step;
    }
    return moved;
}

/* state.rs:130-148 iterate: one tick; returns the summed |step|. */
double orc_fa2_iterate(orc_fa2 *s) {
    orc_fa2_accumulate(s, 7);
    double sw, tr;
    swing_traction(s, &sw, &tr);
    s->swing += sw;
    s->traction += tr;
    estimate_factor(s, s->swing, s->traction);
    s->iter_no++;
    return apply_update(s);
}

/* state.rs:122-128 run: up to `ticks`, stopping once the step sums below 1e-10.
 * Returns the ticks taken. */
uint32_t orc_fa2_run(orc_fa2 *s, uint32_t ticks) {
    uint32_t t = 0;
    while (t < ticks) {
        t++;
        if (orc_fa2_iterate(s) < 1e-10) break;
    }
    return t;
}

/* Row-major n x dim copies in and out of the state. */
void orc_fa2_get_positions(const orc_fa2 *s, double *out) {
    for (uint32_t i = 0; i < s->n; i++)
        for (int a = 0; a < s->dim; a++) out[(size_t)i * s->dim + a] = s->p[(size_t)i * MAXD + a];
}

void orc_fa2_set_positions(orc_fa2 *s, const double *in) {
    for (uint32_t i = 0; i < s->n; i++)
        for (int a = 0; a < s->dim; a++) s->p[(size_t)i * MAXD + a] = in[(size_t)i * s->dim + a];
}

void orc_fa2_get_forces(const orc_fa2 *s, double *out) {
    for (uint32_t i = 0; i < s->n; i++)
        for (int a = 0; a < s->dim; a++) out[(size_t)i * s->dim + a] = s->u[(size_t)i * MAXD + a];
}

void orc_fa2_get_mass(const orc_fa2 *s, double *out) {
    for (uint32_t i = 0; i < s->n; i++) out[i] = s->mass[i];
}

/* swing, traction, speed, speed_efficiency, iter_no, far and pair interaction
 * counts since the state was made. */
void orc_fa2_get_scalars(const orc_fa2 *s, double *out) {
    out[0] = s->swing;
    out[1] = s->traction;
    out[2] = s->speed;
    out[3] = s->speed_efficiency;
    out[4] = (double)s->iter_no;
    out[5] = (double)s->far_count;
    out[6] = (double)s->pair_count;
}

void orc_fa2_set_scalars(orc_fa2 *s, const double *in) {
    s->swing = in[0];
    s->traction = in[1];
    s->speed = in[2];
    s->speed_efficiency = in[3];
    s->iter_no = (uint32_t)in[4];
}

/* The last tree built: cell count, and per cell its width and subtree skip;
 * per point its place in `order`. For structure checks against the GPU tree. */
uint32_t orc_fa2_tree_cells(const orc_fa2 *s) { return (uint32_t)s->tree.ncells; }

void orc_fa2_tree_dump(const orc_fa2 *s, double *width, uint32_t *skip, uint32_t *start,
                       uint32_t *end, double *mass, double *com, uint32_t *order) {
    const ttree *t = &s->tree;
    for (size_t k = 0; k < t->ncells; k++) {
        if (width) width[k] = t->cells[k].b1[0] - t->cells[k].b0[0];
        if (skip) skip[k] = t->cells[k].skip;
        if (start) start[k] = t->cells[k].start;
        if (end) end[k] = t->cells[k].end;
        if (mass) mass[k] = t->bodies ? t->bodies[k].mass : 0.0;
        if (com)
            for (int a = 0; a < s->dim; a++) com[k * s->dim + a] = t->bodies ? t->bodies[k].c[a] : 0.0;
    }
    if (order)
        for (size_t q = 0; q < t->norder; q++) order[q] = t->order[q];
}

/* gravity's own mean, for the association pin (state/tests.rs:27-62). */
void orc_fa2_mean(const orc_fa2 *s, double *out) {
    double mean[MAXD];
    pos_mean(s, mean);
    for (int a = 0; a < s->dim; a++) out[a] = mean[a];
}

/* repel_delta on its own (state/tests.rs:69-94). */
void orc_fa2_repel_delta(const orc_fa2 *s, uint32_t i, uint32_t j, double *out) {
    double dl[MAXD];
    repel_delta(s, i, j, dl);
    for (int a = 0; a < s->dim; a++) out[a] = dl[a];
}

/* ------------------------------------------------------------ adjoint --- */
/*
 * The vector-Jacobian product of a run of ticks (no counterpart in the
 * reference, which has no gradient): the exact derivative of iterate()
 * (state.rs:130-148) with respect to the positions and the attraction
 * coefficients, through the tree each tick built (its far / pair decisions are
 * held fixed; cell centres still move with the points) and through the speed
 * controller on its active branch (estimate_factor's comparisons held fixed).
 * The coincident-pair jiggle is a constant and contributes nothing.
 */

typedef struct {
    double SW, TR, speed, se;
    uint32_t iter;
} ctrl;

/* estimate_factor on explicit state, also returning its partial derivatives:
 * d[0..3] = d speed'/d(SW, TR, speed, se), d[4] = d se'/d se. */
static void ef_diff(double n, double jt, const ctrl *in, double *speed_out, double *se_out, double *d) {
    const double SW = in->SW, TR = in->TR;
    const double opt = 0.05 * sqrt(n), minj = sqrt(opt);
    const double ratio = opt * TR / (n * n);
    double other = ratio < 10.0 ? ratio : 10.0;
    double djit_dTR = 0.0;
    double jitter;
    if (minj >= other) {
        jitter = jt * minj;
    } else {
        jitter = jt * other;
        if (ratio < 10.0) djit_dTR = jt * opt / (n * n);
    }
    double se = in->se, k1 = 1.0;
    if (SW / TR > 2.0) {
        if (se > 0.05) k1 = 0.5;
        if (jt > jitter) {
            jitter = jt;
            djit_dTR = 0.0;
        }
    }
    const double se1 = se * k1;
    double target = INFINITY, dt_dSW = 0.0, dt_dTR = 0.0, dt_dse = 0.0;
    if (SW != 0.0) {
        target = jitter * se1 * TR / SW;
        dt_dSW = -target / SW;
        dt_dTR = jitter * se1 / SW + se1 * TR / SW * djit_dTR;
        dt_dse = jitter * k1 * TR / SW;
    }
    double k2 = 1.0;
    if (SW > jitter * TR) {
        if (se1 > 0.05) k2 = 0.7;
    } else if (in->speed < 1000.0) {
        k2 = 1.3;
    }
    *se_out = se1 * k2;
    d[4] = k1 * k2;
    const double sp = in->speed;
    if (target - sp < 0.5 * sp) {
        *speed_out = sp + (target - sp);
        d[0] = dt_dSW;
        d[1] = dt_dTR;
        d[2] = 0.0;
        d[3] = dt_dse;
    } else {
        *speed_out = sp + 0.5 * sp;
        d[0] = d[1] = d[3] = 0.0;
        d[2] = 1.5;
    }
}

/* d (k m_i M d / |d|^2) / d d, applied to v: k m_i M (v/|d|^2 - 2 d (d.v)/|d|^4). */
static void rep_jac(int dim, double coef, const double *dl, const double *v, double *out) {
    double d2 = norm2(dl, dim), dv = 0.0;
    for (int a = 0; a < dim; a++) dv += dl[a] * v[a];
    for (int a = 0; a < dim; a++) out[a] = coef * (v[a] / d2 - 2.0 * dl[a] * dv / (d2 * d2));
}

/* Adjoint of one tick at the state's current positions and controller `c`
 * (the values before the tick). In: lam1 = dL/dp', L1 = adjoint of the
 * controller after the tick (SW', TR', speed', se'). Out: lam0 = dL/dp,
 * L0 = adjoint of the controller before, gc += dL/dc per simple edge. */
static void tick_adjoint(orc_fa2 *s, const ctrl *c, const double *lam1, const double *L1, double *lam0, double *L0,
                         double *gc) {
    const int d = s->dim;
    const uint32_t n = s->n;
    const double N = (double)n;
    s->iter_no = c->iter;
    orc_fa2_accumulate(s, 7); /* u at these positions, and this tick's tree */
    double sw = 0.0, tr = 0.0;
    swing_traction(s, &sw, &tr);
    ctrl after = {c->SW + sw, c->TR + tr, c->speed, c->se, c->iter};
    double speed1, se1, dd[5];
    ef_diff(N, s->P.jitter_tolerance, &after, &speed1, &se1, dd);
    double *ub = (double *)calloc((size_t)n * MAXD, sizeof(double));
    /* update: p' = p + f u, f = speed1 / (1 + sqrt(speed1 m |u|)) */
    double Lsp = L1[2];
    for (uint32_t i = 0; i < n; i++) {
        const double *u = s->u + (size_t)i * MAXD, *l = lam1 + (size_t)i * d;
        double un = sqrt(norm2(u, d)), m = s->mass[i];
        double q = sqrt(speed1 * m * un), f = speed1 / (1.0 + q);
        double lu = 0.0;
        for (int a = 0; a < d; a++) lu += l[a] * u[a];
        double dfds = q > 0.0 ? (1.0 + 0.5 * q) / ((1.0 + q) * (1.0 + q)) : 1.0;
        Lsp += lu * dfds;
        for (int a = 0; a < d; a++) {
            lam0[(size_t)i * d + a] = l[a];
            ub[(size_t)i * MAXD + a] = f * l[a];
        }
        if (q > 0.0) { /* grad_u f = -speed1/(1+q)^2 * speed1 m u / (2 q |u|) */
            double g = -speed1 / ((1.0 + q) * (1.0 + q)) * speed1 * m / (2.0 * q * un);
            for (int a = 0; a < d; a++) ub[(size_t)i * MAXD + a] += lu * g * u[a];
        }
    }
    /* controller: speed1 = EF(SW', TR', speed, se), se1 likewise */
    const double Lse = L1[3];
    double LSW = L1[0] + Lsp * dd[0], LTR = L1[1] + Lsp * dd[1];
    L0[2] = Lsp * dd[2];
    L0[3] = Lsp * dd[3] + Lse * dd[4];
    L0[0] = LSW;
    L0[1] = LTR;
    /* swing = sum m |p - u|, traction = sum 0.5 m |p + u| */
    for (uint32_t i = 0; i < n; i++) {
        const double *p = s->p + (size_t)i * MAXD, *u = s->u + (size_t)i * MAXD;
        double b[MAXD], g[MAXD], m = s->mass[i];
        for (int a = 0; a < d; a++) {
            b[a] = p[a] - u[a];
            g[a] = p[a] + u[a];
        }
        double bn = sqrt(norm2(b, d)), gn = sqrt(norm2(g, d));
        for (int a = 0; a < d; a++) {
            double tb = bn > 0.0 ? LSW * m * b[a] / bn : 0.0;
            double tg = gn > 0.0 ? LTR * 0.5 * m * g[a] / gn : 0.0;
            lam0[(size_t)i * d + a] += tb + tg;
            ub[(size_t)i * MAXD + a] += -tb + tg;
        }
    }
    /* gravity: g_i = -gm c/|c| (or -gm c), c = p - mean */
    {
        double vmean[MAXD] = {0, 0, 0};
        double *v = (double *)calloc((size_t)n * MAXD, sizeof(double));
        double mean[MAXD];
        pos_mean(s, mean);
        for (uint32_t i = 0; i < n; i++) {
            double cc[MAXD], gm = s->P.gravity * s->mass[i];
            const double *ui = ub + (size_t)i * MAXD;
            for (int a = 0; a < d; a++) cc[a] = s->p[(size_t)i * MAXD + a] - mean[a];
            double *vi = v + (size_t)i * MAXD;
            if (s->P.strong_gravity) {
                for (int a = 0; a < d; a++) vi[a] = -gm * ui[a];
            } else {
                double cn = sqrt(norm2(cc, d));
                if (cn > 0.0) {
                    double cu = 0.0;
                    for (int a = 0; a < d; a++) cu += cc[a] * ui[a];
                    for (int a = 0; a < d; a++) vi[a] = -gm * (ui[a] - cc[a] * cu / (cn * cn)) / cn;
                }
            }
            for (int a = 0; a < d; a++) vmean[a] += vi[a];
        }
        for (int a = 0; a < d; a++) vmean[a] /= N;
        for (uint32_t i = 0; i < n; i++)
            for (int a = 0; a < d; a++) lam0[(size_t)i * d + a] += v[(size_t)i * MAXD + a] - vmean[a];
        free(v);
    }
    /* attraction: a_i = sum_j c phi(|delta|) delta, delta = p_j - p_i; u_i += a_i (/ m_i) */
    for (int64_t e = 0; e < s->m; e++) {
        uint32_t i = s->lo[e], j = s->hi[e];
        double dl[MAXD], ai[MAXD], aj[MAXD];
        double mi = s->P.dissuade_hubs ? s->mass[i] : 1.0, mj = s->P.dissuade_hubs ? s->mass[j] : 1.0;
        for (int a = 0; a < d; a++) {
            dl[a] = s->p[(size_t)j * MAXD + a] - s->p[(size_t)i * MAXD + a];
            ai[a] = ub[(size_t)i * MAXD + a] / mi;
            aj[a] = ub[(size_t)j * MAXD + a] / mj;
        }
        double dist = sqrt(norm2(dl, d));
        double phi = 1.0, dphi = 0.0;
        if (s->P.lin_log) {
            if (dist > 0.0) {
                phi = log(1.0 + dist) / dist;
                dphi = (dist / (1.0 + dist) - log(1.0 + dist)) / (dist * dist);
            } else {
                phi = 0.0; /* the forward's zero-distance convention */
            }
        }
        double cw = s->w[e];
        double diff[MAXD], ddot = 0.0;
        for (int a = 0; a < d; a++) {
            diff[a] = aj[a] - ai[a];
            ddot += dl[a] * diff[a];
        }
        /* lam_j += J (a_j - a_i)... J = c (phi I + dphi delta delta^T / dist) */
        for (int a = 0; a < d; a++) {
            double jv = cw * (phi * diff[a] + (dist > 0.0 ? dphi * dl[a] * ddot / dist : 0.0));
            lam0[(size_t)j * d + a] -= jv;
            lam0[(size_t)i * d + a] += jv;
        }
        double g = 0.0;
        for (int a = 0; a < d; a++) g += phi * (ai[a] - aj[a]) * dl[a];
        gc[e] += g;
    }
    /* repulsion */
    const double kr = s->P.scaling_ratio;
    if (s->P.theta < 0.0) {
        for (uint32_t i = 0; i < n; i++)
            for (uint32_t j = i + 1; j < n; j++) {
                double dl[MAXD], v[MAXD], out[MAXD];
                int zero = 1;
                for (int a = 0; a < d; a++) {
                    dl[a] = s->p[(size_t)i * MAXD + a] - s->p[(size_t)j * MAXD + a];
                    if (dl[a] != 0.0) zero = 0;
                    v[a] = ub[(size_t)i * MAXD + a] - ub[(size_t)j * MAXD + a];
                }
                if (zero) continue;
                rep_jac(d, kr * s->mass[i] * s->mass[j], dl, v, out);
                for (int a = 0; a < d; a++) {
                    lam0[(size_t)i * d + a] += out[a];
                    lam0[(size_t)j * d + a] -= out[a];
                }
            }
    } else {
        ttree *t = &s->tree;
        double th2 = s->P.theta * s->P.theta;
        double *cbar = (double *)calloc(t->ncells * MAXD + 1, sizeof(double));
        for (size_t p = 0; p < t->norder; p++) {
            uint32_t i = t->order[p];
            const double *xi = s->p + (size_t)i * MAXD, *ui = ub + (size_t)i * MAXD;
            double mi = s->mass[i];
            size_t k = 0;
            while (k < t->ncells) {
                const tcell *cl = &t->cells[k];
                int holds = cl->start <= p && p < cl->end;
                const tbody *b = &t->bodies[k];
                double dl[MAXD];
                for (int a = 0; a < d; a++) dl[a] = xi[a] - b->c[a];
                double d2 = norm2(dl, d), w = cl->b1[0] - cl->b0[0];
                if (!holds && d2 > 0.0 && w * w < th2 * d2) {
                    double out[MAXD];
                    rep_jac(d, kr * mi * b->mass, dl, ui, out);
                    for (int a = 0; a < d; a++) {
                        lam0[(size_t)i * d + a] += out[a];
                        cbar[k * MAXD + a] -= out[a];
                    }
                    k = cl->skip;
                } else if (cl->skip == k + 1) {
                    for (uint32_t q = cl->start; q < cl->end; q++) {
                        uint32_t j = t->order[q];
                        if (j == i) continue;
                        double dj[MAXD], out[MAXD];
                        int zero = 1;
                        for (int a = 0; a < d; a++) {
                            dj[a] = xi[a] - s->p[(size_t)j * MAXD + a];
                            if (dj[a] != 0.0) zero = 0;
                        }
                        if (zero) continue;
                        rep_jac(d, kr * mi * s->mass[j], dj, ui, out);
                        for (int a = 0; a < d; a++) {
                            lam0[(size_t)i * d + a] += out[a];
                            lam0[(size_t)j * d + a] -= out[a];
                        }
                    }
                    k++;
                } else {
                    k++;
                }
            }
        }
        /* a cell centre is sum m_j p_j / M over its points */
        for (size_t k = 0; k < t->ncells; k++) {
            const tcell *cl = &t->cells[k];
            double M = t->bodies[k].mass;
            for (uint32_t q = cl->start; q < cl->end; q++) {
                uint32_t j = t->order[q];
                for (int a = 0; a < d; a++) lam0[(size_t)j * d + a] += s->mass[j] / M * cbar[k * MAXD + a];
            }
        }
        free(cbar);
    }
    free(ub);
}

/* Runs `ticks` ticks from the current state, recording each tick's positions
 * and controller, then pulls lamT = dL/d(final positions) (n x dim) back:
 * lam0 = dL/d(start positions) (n x dim), gc = dL/d(attraction coefficient) per
 * simple edge (the caller multiplies by dc/dw). The state ends at the final
 * positions. */
void orc_fa2_adjoint(orc_fa2 *s, uint32_t ticks, const double *lamT, double *lam0, double *gc) {
    const int d = s->dim;
    const uint32_t n = s->n;
    double *hist = (double *)malloc(((size_t)ticks + 1) * n * MAXD * sizeof(double) + 8);
    ctrl *cs = (ctrl *)malloc(((size_t)ticks + 1) * sizeof(ctrl));
    for (uint32_t t = 0; t < ticks; t++) {
        memcpy(hist + (size_t)t * n * MAXD, s->p, (size_t)n * MAXD * sizeof(double));
        cs[t] = (ctrl){s->swing, s->traction, s->speed, s->speed_efficiency, s->iter_no};
        orc_fa2_iterate(s);
    }
    double *lam = (double *)malloc((size_t)n * d * sizeof(double) + 8);
    double *nxt = (double *)malloc((size_t)n * d * sizeof(double) + 8);
    memcpy(lam, lamT, (size_t)n * d * sizeof(double));
    double L1[4] = {0, 0, 0, 0}, L0[4];
    for (int64_t e = 0; e < s->m; e++) gc[e] = 0.0;
    double *keep = (double *)malloc((size_t)n * MAXD * sizeof(double) + 8);
    memcpy(keep, s->p, (size_t)n * MAXD * sizeof(double));
    ctrl last = {s->swing, s->traction, s->speed, s->speed_efficiency, s->iter_no};
    for (uint32_t t = ticks; t-- > 0;) {
        memcpy(s->p, hist + (size_t)t * n * MAXD, (size_t)n * MAXD * sizeof(double));
        tick_adjoint(s, &cs[t], lam, L1, nxt, L0, gc);
        memcpy(lam, nxt, (size_t)n * d * sizeof(double));
        memcpy(L1, L0, sizeof L1);
    }
    memcpy(lam0, lam, (size_t)n * d * sizeof(double));
    memcpy(s->p, keep, (size_t)n * MAXD * sizeof(double));
    s->swing = last.SW;
    s->traction = last.TR;
    s->speed = last.speed;
    s->speed_efficiency = last.se;
    s->iter_no = last.iter;
    free(keep);
    free(lam);
    free(nxt);
    free(hist);
    free(cs);
}

/* The simple edges' attraction coefficients (w^influence), in / out. */
void orc_fa2_get_coef(const orc_fa2 *s, double *out) {
    for (int64_t e = 0; e < s->m; e++) out[e] = s->w[e];
}
void orc_fa2_set_coef(orc_fa2 *s, const double *in) {
    for (int64_t e = 0; e < s->m; e++) s->w[e] = in[e];
}


/* ------------------------------------------------------------- stress ------ */

/* Adjacency of the raw edges as graph-cli/src/bench.rs:258-262 builds it: for
 * edge (s, t) in edge order, t is pushed to s's list and s to t's (a self-loop
 * appears twice in its own list). */
static void stress_adjacency(uint32_t n, uint64_t m, const uint32_t *src, const uint32_t *dst, uint64_t **rp_out,
                             uint32_t **adj_out) {
    uint64_t *rp = (uint64_t *)calloc((size_t)n + 1, sizeof(uint64_t));
    for (uint64_t e = 0; e < m; e++) {
        rp[src[e] + 1]++;
        rp[dst[e] + 1]++;
    }
    for (uint32_t i = 0; i < n; i++) rp[i + 1] += rp[i];
    uint32_t *adj = (uint32_t *)malloc((size_t)(rp[n] ? rp[n] : 1) * sizeof(uint32_t));
    uint64_t *fill = (uint64_t *)malloc((size_t)(n ? n : 1) * sizeof(uint64_t));
    for (uint32_t i = 0; i < n; i++) fill[i] = rp[i];
    for (uint64_t e = 0; e < m; e++) {
        adj[fill[src[e]]++] = dst[e];
        adj[fill[dst[e]]++] = src[e];
    }
    free(fill);
    *rp_out = rp;
    *adj_out = adj;
}

/* One FIFO BFS (bench.rs:267-277): hop[v] = UINT32_MAX when unreachable. */
static void stress_bfs(uint32_t n, const uint64_t *rp, const uint32_t *adj, uint32_t from, uint32_t *hop,
                       uint32_t *queue) {
    for (uint32_t i = 0; i < n; i++) hop[i] = UINT32_MAX;
    uint32_t head = 0, tail = 0;
    hop[from] = 0;
    queue[tail++] = from;
    while (head < tail) {
        uint32_t v = queue[head++];
        for (uint64_t e = rp[v]; e < rp[v + 1]; e++) {
            uint32_t w = adj[e];
            if (hop[w] == UINT32_MAX) {
                hop[w] = hop[v] + 1;
                queue[tail++] = w;
            }
        }
    }
}

/* graph-cli/src/bench.rs:255-295 `stress`: BFS from every max(n / sources, 1)-th
 * node; per reachable target in ascending order d = hops, e = hypot((f64)(x[to] -
 * x[from]), (f64)(y[to] - y[from])) with the difference taken in f32; DE, EE, DD
 * summed in that order; sqrt(max((DD - DE / EE * DE) / DD, 0)), or 1 when EE or DD
 * is 0. */
double orc_stress(uint32_t n, uint64_t m, const uint32_t *src, const uint32_t *dst, const float *x, const float *y,
                  uint32_t sources) {
    if (n == 0) return 1.0;
    uint64_t *rp;
    uint32_t *adj;
    stress_adjacency(n, m, src, dst, &rp, &adj);
    uint32_t *hop = (uint32_t *)malloc((size_t)n * sizeof(uint32_t));
    uint32_t *queue = (uint32_t *)malloc((size_t)n * sizeof(uint32_t));
    double de = 0.0, ee = 0.0, dd = 0.0;
    uint32_t step = n / sources;
    if (step < 1) step = 1;
    for (uint64_t from = 0; from < n; from += step) {
        stress_bfs(n, rp, adj, (uint32_t)from, hop, queue);
        for (uint32_t to = 0; to < n; to++) {
            if (to == from || hop[to] == UINT32_MAX) continue;
            double dist = (double)hop[to];
            double dx = (double)(x[to] - x[from]), dy = (double)(y[to] - y[from]);
            double euclid = hypot(dx, dy);
            de += dist * euclid;
            ee += euclid * euclid;
            dd += dist * dist;
        }
    }
    free(queue);
    free(hop);
    free(adj);
    free(rp);
    if (ee == 0.0 || dd == 0.0) return 1.0;
    double r = (dd - de / ee * de) / dd;
    return sqrt(r > 0.0 ? r : 0.0);
}

/* Hop counts from each of k sources by the same BFS (out: k x n). */
void orc_bfs(uint32_t n, uint64_t m, const uint32_t *src, const uint32_t *dst, uint32_t k, const uint32_t *sources,
             uint32_t *out) {
    if (n == 0) return;
    uint64_t *rp;
    uint32_t *adj;
    stress_adjacency(n, m, src, dst, &rp, &adj);
    uint32_t *queue = (uint32_t *)malloc((size_t)n * sizeof(uint32_t));
    for (uint32_t j = 0; j < k; j++) stress_bfs(n, rp, adj, sources[j], out + (size_t)j * n, queue);
    free(queue);
    free(adj);
    free(rp);
}


/* ============================================== d3-force Barnes-Hut ======= */
/*
 * The frozen d3-force layout of graph-core (crates/graph-core/src/layout/force/
 * barnes_hut.rs, barnes_hut/{sim,seed,link,charge,collide}.rs, charge/{aggregate,
 * threshold}.rs, params.rs, session.rs), restated in FP64 in the reference's
 * operation order: golden-spiral start, then per tick alpha decay, link (Jacobi:
 * every edge's force from the tick's state, then each node's shares in its row's
 * order), many-body over the insertion quadtree of the positions (cell bodies in
 * reverse preorder, the stackless walk with d3's `open >= l` test, distanceMin /
 * distanceMax, jiggle keyed on the cell's arena index), center, collide over the
 * quadtree of the projected positions, integrate. Each pass adds one delta per
 * node to its velocity.
 */

typedef struct {
    double charge, theta, distance_min, distance_max, link_distance, link_strength_scale, collide_radius,
        center_strength, velocity_decay, alpha_decay, alpha_min, initial_alpha;
} orc_d3_params;

typedef struct {
    double comx, comy, open;
    uint32_t count, skip, start;
} d3body;

typedef struct {
    orc_d3_params P;
    uint32_t n, m, seed, tick_no;
    double alpha;
    uint32_t *lo, *hi;
    double *dist, *stren, *bias;
    uint32_t *rp, *rows; /* node -> its simple edges, ascending edge index */
    double *x, *y, *vx, *vy, *px, *py, *pos, *dvx, *dvy, *fx, *fy;
    ttree ct, kt; /* charge tree, collide tree */
    d3body *bodies;
    int mesh;       /* many-body on the particle mesh (particle_mesh.rs) instead of the tree */
    uint32_t side;  /* mesh side (mesh.rs side_for) */
    double *gre, *gim, *kre, *kim, *twr, *twi; /* density/field, kernel spectrum, twiddles */
} orc_d3;

/* seed.rs spiral_point: radius 12 sqrt(i + 1), angle i * golden angle. */
static void d3_spiral(uint32_t i, double *x, double *y) {
    const double golden = 2.399963229728653;
    double radius = 12.0 * sqrt((double)i + 1.0);
    double angle = (double)i * golden;
    *x = cos(angle) * radius;
    *y = sin(angle) * radius;
}

/* params.rs:60-75 defaults (the production engine's values). */
void orc_d3_default_params(orc_d3_params *p) {
    p->charge = -90.0;
    p->theta = 0.9;
    p->distance_min = 1.0;
    p->distance_max = 520.0;
    p->link_distance = 60.0;
    p->link_strength_scale = 0.15;
    p->collide_radius = 16.0;
    p->center_strength = 1.0;
    p->velocity_decay = 1.0 - 0.42;
    p->alpha_decay = 0.06;
    p->alpha_min = 0.001;
    p->initial_alpha = 1.0;
}

/* Sim::new over the simple graph (lo < hi, first-wins strength, edge order). A
 * null pos0 starts from the golden spiral (seed.rs golden_spiral). */
orc_d3 *orc_d3_new(uint32_t n, uint32_t m, const uint32_t *lo, const uint32_t *hi, const double *strength,
                   const orc_d3_params *P, const double *pos0) {
    orc_d3 *s = (orc_d3 *)calloc(1, sizeof(orc_d3));
    s->P = *P;
    s->n = n;
    s->m = m;
    s->alpha = P->initial_alpha;
    size_t nn = n ? n : 1, mm = m ? m : 1;
    s->lo = (uint32_t *)malloc(mm * 4);
    s->hi = (uint32_t *)malloc(mm * 4);
    s->dist = (double *)malloc(mm * 8);
    s->stren = (double *)malloc(mm * 8);
    s->bias = (double *)malloc(mm * 8);
    s->fx = (double *)malloc(mm * 8);
    s->fy = (double *)malloc(mm * 8);
    memcpy(s->lo, lo, (size_t)m * 4);
    memcpy(s->hi, hi, (size_t)m * 4);
    /* mod.rs:177-180 row_csr: (lo[e], e), (hi[e], e) in edge order */
    s->rp = (uint32_t *)calloc(nn + 1, 4);
    for (uint32_t e = 0; e < m; e++) {
        s->rp[lo[e] + 1]++;
        s->rp[hi[e] + 1]++;
    }
    for (uint32_t i = 0; i < n; i++) s->rp[i + 1] += s->rp[i];
    s->rows = (uint32_t *)malloc((2 * (size_t)m + 1) * 4);
    uint32_t *fill = (uint32_t *)malloc(nn * 4);
    for (uint32_t i = 0; i < n; i++) fill[i] = s->rp[i];
    for (uint32_t e = 0; e < m; e++) {
        s->rows[fill[lo[e]]++] = e;
        s->rows[fill[hi[e]]++] = e;
    }
    free(fill);
    /* link.rs edge_geometry: distance, strength, degree bias */
    for (uint32_t e = 0; e < m; e++) {
        double st = strength[e];
        double dlo = (double)(s->rp[lo[e] + 1] - s->rp[lo[e]]), dhi = (double)(s->rp[hi[e] + 1] - s->rp[hi[e]]);
        s->dist[e] = P->link_distance / fmax(0.4, st);
        s->stren[e] = fmin(0.7, P->link_strength_scale * st);
        s->bias[e] = dlo / (dlo + dhi);
    }
    s->x = (double *)malloc(nn * 8);
    s->y = (double *)malloc(nn * 8);
    s->vx = (double *)calloc(nn, 8);
    s->vy = (double *)calloc(nn, 8);
    s->px = (double *)calloc(nn, 8);
    s->py = (double *)calloc(nn, 8);
    s->dvx = (double *)calloc(nn, 8);
    s->dvy = (double *)calloc(nn, 8);
    s->pos = (double *)calloc(nn * MAXD, 8);
    for (uint32_t i = 0; i < n; i++) {
        if (pos0) {
            s->x[i] = pos0[2 * i];
            s->y[i] = pos0[2 * i + 1];
        } else {
            d3_spiral(i, &s->x[i], &s->y[i]);
        }
    }
    return s;
}

void orc_d3_free(orc_d3 *s) {
    if (!s) return;
    ttree *ts[2] = {&s->ct, &s->kt};
    for (int k = 0; k < 2; k++) {
        free(ts[k]->shape);
        free(ts[k]->chain_next);
        free(ts[k]->cells);
        free(ts[k]->node_id);
        free(ts[k]->order);
        free(ts[k]->bodies);
    }
    free(s->bodies);
    free(s->gre);
    free(s->gim);
    free(s->kre);
    free(s->kim);
    free(s->twr);
    free(s->twi);
    free(s->lo);
    free(s->hi);
    free(s->dist);
    free(s->stren);
    free(s->bias);
    free(s->fx);
    free(s->fy);
    free(s->rp);
    free(s->rows);
    free(s->x);
    free(s->y);
    free(s->vx);
    free(s->vy);
    free(s->px);
    free(s->py);
    free(s->dvx);
    free(s->dvy);
    free(s->pos);
    free(s);
}

static void d3_tree(orc_d3 *s, ttree *t, const double *x, const double *y) {
    for (uint32_t i = 0; i < s->n; i++) {
        s->pos[(size_t)i * MAXD] = x[i];
        s->pos[(size_t)i * MAXD + 1] = y[i];
    }
    tree_build(t, s->pos, s->n, 2, 0);
}

/* link.rs force / share + step.rs LinkPass::node_share + merge. */
static void d3_link(orc_d3 *s) {
    for (uint32_t e = 0; e < s->m; e++) {
        uint32_t lo = s->lo[e], hi = s->hi[e];
        double dx = (s->x[hi] + s->vx[hi]) - (s->x[lo] + s->vx[lo]);
        double dy = (s->y[hi] + s->vy[hi]) - (s->y[lo] + s->vy[lo]);
        if (dx == 0.0) dx = orc_jiggle(s->seed, s->tick_no, 0, lo, hi);
        if (dy == 0.0) dy = orc_jiggle(s->seed, s->tick_no, 1, lo, hi);
        double l = sqrt(dx * dx + dy * dy);
        if (l == 0.0) {
            s->fx[e] = s->fy[e] = 0.0;
            continue;
        }
        double factor = (l - s->dist[e]) / l * s->alpha * s->stren[e];
        s->fx[e] = dx * factor;
        s->fy[e] = dy * factor;
    }
    for (uint32_t v = 0; v < s->n; v++) {
        double ax = 0.0, ay = 0.0;
        for (uint32_t q = s->rp[v]; q < s->rp[v + 1]; q++) {
            uint32_t e = s->rows[q];
            double b = s->bias[e];
            if (s->hi[e] == v) {
                ax += -s->fx[e] * b;
                ay += -s->fy[e] * b;
            } else {
                ax += s->fx[e] * (1.0 - b);
                ay += s->fy[e] * (1.0 - b);
            }
        }
        s->vx[v] += ax;
        s->vy[v] += ay;
    }
}

/* threshold.rs opening_threshold. */
static double d3_open(double w, double theta, double theta2) {
    if (theta == 0.0) return INFINITY;
    double naive = w * w / theta2;
    if (!isnan(naive)) return naive;
    if (!isfinite(theta)) return INFINITY;
    double ratio = w / theta;
    return isfinite(ratio) ? ratio * ratio : INFINITY;
}

/* charge.rs settle: 0 past distanceMax, a zero axis jiggled (passes 2, 3), l
 * clamped up to distanceMin. Returns 0 when the term is dropped. */
static int d3_settle(const orc_d3 *s, uint32_t i, uint32_t key, double *dx, double *dy, double *l) {
    double dmin2 = s->P.distance_min * s->P.distance_min, dmax2 = s->P.distance_max * s->P.distance_max;
    if (*l >= dmax2) return 0;
    if (*dx == 0.0) {
        *dx = orc_jiggle(s->seed, s->tick_no, 2, i, key);
        *l += *dx * *dx;
    }
    if (*dy == 0.0) {
        *dy = orc_jiggle(s->seed, s->tick_no, 3, i, key);
        *l += *dy * *dy;
    }
    if (*l < dmin2) *l = sqrt(dmin2 * *l);
    if (*l == 0.0) *l = dmin2 > DBL_MIN_POS ? dmin2 : DBL_MIN_POS;
    return 1;
}

/* charge.rs: aggregate (reverse preorder) then node_delta for every node. */
static void d3_charge(orc_d3 *s) {
    ttree *t = &s->ct;
    d3_tree(s, t, s->x, s->y);
    size_t nc = t->ncells;
    s->bodies = (d3body *)realloc(s->bodies, (nc ? nc : 1) * sizeof(d3body));
    double theta = s->P.theta, theta2 = theta * theta;
    for (size_t kk = nc; kk-- > 0;) {
        const tcell *c = &t->cells[kk];
        double cx, cy;
        if (c->skip == kk + 1) {
            uint32_t head = t->order[c->start];
            cx = s->x[head];
            cy = s->y[head];
        } else {
            double m = 0.0, sx = 0.0, sy = 0.0;
            for (uint32_t ch = (uint32_t)kk + 1; ch < c->skip; ch = s->bodies[ch].skip) {
                double cm = (double)s->bodies[ch].count;
                m += cm;
                sx += cm * s->bodies[ch].comx;
                sy += cm * s->bodies[ch].comy;
            }
            cx = sx / m;
            cy = sy / m;
        }
        d3body *b = &s->bodies[kk];
        b->comx = cx;
        b->comy = cy;
        b->open = d3_open(c->b1[0] - c->b0[0], theta, theta2);
        b->count = c->end - c->start;
        b->skip = c->skip;
        b->start = c->start;
    }
    double ca = s->P.charge * s->alpha;
    for (uint32_t i = 0; i < s->n; i++) {
        double xi = s->x[i], yi = s->y[i], ox = 0.0, oy = 0.0;
        uint32_t k = 0;
        while (k < nc) {
            const d3body *b = &s->bodies[k];
            double dx = b->comx - xi, dy = b->comy - yi;
            double l = dx * dx + dy * dy;
            double ddx = 0.0, ddy = 0.0;
            uint32_t next;
            if (b->open >= l) {
                if (b->skip != k + 1) {
                    k++;
                    continue;
                }
                const uint32_t *chain = t->order + b->start;
                if (d3_settle(s, i, chain[0], &dx, &dy, &l)) {
                    for (uint32_t q = 0; q < b->count; q++) {
                        if (chain[q] == i) continue;
                        double f = s->P.charge * s->alpha / l;
                        ddx += dx * f;
                        ddy += dy * f;
                    }
                }
                next = k + 1;
            } else {
                if (d3_settle(s, i, (uint32_t)t->node_id[k], &dx, &dy, &l)) {
                    double m = (double)b->count;
                    double f = m * s->P.charge * s->alpha / l;
                    ddx = dx * f;
                    ddy = dy * f;
                }
                next = b->skip;
            }
            ox += ddx;
            oy += ddy;
            k = next;
        }
        s->dvx[i] = ox;
        s->dvy[i] = oy;
    }
    (void)ca;
    for (uint32_t i = 0; i < s->n; i++) {
        s->vx[i] += s->dvx[i];
        s->vy[i] += s->dvy[i];
    }
}

/* sim.rs center / center_shift. */
static void d3_center(orc_d3 *s) {
    if (s->n == 0) return;
    double sx = 0.0, sy = 0.0;
    for (uint32_t i = 0; i < s->n; i++) {
        sx += s->x[i];
        sy += s->y[i];
    }
    double dx = (sx / (double)s->n) * s->P.center_strength, dy = (sy / (double)s->n) * s->P.center_strength;
    for (uint32_t i = 0; i < s->n; i++) {
        s->x[i] -= dx;
        s->y[i] -= dy;
    }
}

/* collide.rs: tree over x + vx, every point within 2 r pushed apart by half. */
static void d3_collide(orc_d3 *s) {
    for (uint32_t i = 0; i < s->n; i++) {
        s->px[i] = s->x[i] + s->vx[i];
        s->py[i] = s->y[i] + s->vy[i];
    }
    ttree *t = &s->kt;
    d3_tree(s, t, s->px, s->py);
    double diameter = 2.0 * s->P.collide_radius, d2 = diameter * diameter, reach = sqrt(d2);
    for (uint32_t i = 0; i < s->n; i++) {
        double xi = s->px[i], yi = s->py[i], ox = 0.0, oy = 0.0;
        uint32_t k = 0;
        while (k < t->ncells) {
            const tcell *c = &t->cells[k];
            if (c->skip == k + 1) {
                for (uint32_t q = c->start; q < c->end; q++) {
                    uint32_t p = t->order[q];
                    if (p == i) continue;
                    double dx = xi - s->px[p], dy = yi - s->py[p];
                    double l = dx * dx + dy * dy;
                    if (l >= d2) continue;
                    if (dx == 0.0) {
                        dx = orc_jiggle(s->seed, s->tick_no, 4, i, p);
                        l += dx * dx;
                    }
                    if (dy == 0.0) {
                        dy = orc_jiggle(s->seed, s->tick_no, 5, i, p);
                        l += dy * dy;
                    }
                    double dist = sqrt(l);
                    double push = (reach - dist) / dist * 0.5;
                    ox += dx * push;
                    oy += dy * push;
                }
                k = k + 1;
            } else if (c->b0[0] > xi + reach || c->b1[0] < xi - reach || c->b0[1] > yi + reach ||
                       c->b1[1] < yi - reach) {
                k = c->skip;
            } else {
                k = k + 1;
            }
        }
        s->dvx[i] = ox;
        s->dvy[i] = oy;
    }
    for (uint32_t i = 0; i < s->n; i++) {
        s->vx[i] += s->dvx[i];
        s->vy[i] += s->dvy[i];
    }
}

/* ------------------------------------------------- particle mesh -------- */
/*
 * The many-body pass of graph-core's particle-mesh layout
 * (crates/graph-core/src/layout/force/particle_mesh/{mesh,frame,deposit,kernel,
 * fft,charge}.rs): the positions' bounding box placed on a side x side mesh
 * (frame.rs place / fit: cell size 2^(step/4), the smallest step whose cells +
 * reach fit), cloud-in-cell deposit of unit masses (deposit.rs weights), the
 * law's vector Green's function sampled within reach and scaled by 1/side^2
 * (kernel.rs sample / green: -r/l, l clamped up to distanceMin, nothing at or
 * past distanceMax), one complex FFT convolution (field = re, im), bilinear read
 * at every node, times charge * alpha onto the velocity. The FFT here is a plain
 * radix-2 transform with the reference's sign and normalisation (forward
 * exp(-2 pi i k / N), both directions unscaled).
 */

/* mesh.rs side_for: next power of two of ceil(sqrt(n)), clamped to [128, 1024]. */
static uint32_t pm_side(uint32_t n) {
    uint32_t root = (uint32_t)ceil(sqrt((double)n)), side = 1;
    while (side < root) side <<= 1;
    return side < 128 ? 128 : (side > 1024 ? 1024 : side);
}

typedef struct {
    int step;
    double h, ox, oy;
    uint32_t cells, reach;
} pm_frame;

/* frame.rs fit / place. */
static int pm_place(double lx, double ly, double hx, double hy, uint32_t side, double dmax, pm_frame *f) {
    double span = fmax(hx - lx, hy - ly);
    if (!isfinite(span)) return 0;
    int step = (int)floor(4.0 * log2(span / (double)side));
    if (step < -32) step = -32;
    for (;; step++) {
        double h = exp2((double)step / 4.0);
        double cells = floor(span / h) + 3.0;
        if (cells > (double)side) continue;
        uint32_t c = (uint32_t)cells;
        double rr = ceil(dmax / h);
        uint32_t reach = rr > (double)(c - 1) ? c - 1 : (uint32_t)rr;
        if (c + reach > side) continue;
        f->step = step;
        f->h = h;
        f->cells = c;
        f->reach = reach;
        f->ox = floor(lx / h) * h;
        f->oy = floor(ly / h) * h;
        return 1;
    }
}

/* frame.rs scaled + split: the node's cell and its fractions within it. */
static void pm_split(const pm_frame *f, double px, double py, uint32_t *cx, uint32_t *cy, double *fx, double *fy) {
    double u[2] = {(px - f->ox) / f->h, (py - f->oy) / f->h};
    uint32_t c[2];
    double fr[2];
    for (int a = 0; a < 2; a++) {
        double v = u[a] > 0.0 ? u[a] : 0.0; /* `u as usize` saturates at 0 */
        uint32_t cell = (uint32_t)v;
        if (cell > f->cells - 2) cell = f->cells - 2;
        double t = u[a] - (double)cell;
        fr[a] = t < 0.0 ? 0.0 : (t > 1.0 ? 1.0 : t);
        c[a] = cell;
    }
    *cx = c[0];
    *cy = c[1];
    *fx = fr[0];
    *fy = fr[1];
}

/* One radix-2 line transform (bit reversal, then log2(N) butterfly stages). */
static void pm_line(double *re, double *im, uint32_t N, size_t stride, const double *twr, const double *twi,
                    int inverse) {
    uint32_t bits = 0;
    while ((1u << bits) < N) bits++;
    for (uint32_t i = 0; i < N; i++) {
        uint32_t j = 0;
        for (uint32_t b = 0; b < bits; b++) j |= ((i >> b) & 1u) << (bits - 1 - b);
        if (i < j) {
            double t = re[i * stride];
            re[i * stride] = re[j * stride];
            re[j * stride] = t;
            t = im[i * stride];
            im[i * stride] = im[j * stride];
            im[j * stride] = t;
        }
    }
    for (uint32_t m = 1; m < N; m <<= 1) {
        for (uint32_t g = 0; g < N; g += 2 * m) {
            for (uint32_t k = 0; k < m; k++) {
                uint32_t t = k * (N / (2 * m));
                double wr = twr[t], wi = inverse ? -twi[t] : twi[t];
                size_t i0 = (size_t)(g + k) * stride, i1 = (size_t)(g + k + m) * stride;
                double br = re[i1] * wr - im[i1] * wi, bi = re[i1] * wi + im[i1] * wr;
                re[i1] = re[i0] - br;
                im[i1] = im[i0] - bi;
                re[i0] += br;
                im[i0] += bi;
            }
        }
    }
}

static void pm_fft2(orc_d3 *s, double *re, double *im, int inverse) {
    uint32_t N = s->side;
    for (uint32_t r = 0; r < N; r++) pm_line(re + (size_t)r * N, im + (size_t)r * N, N, 1, s->twr, s->twi, inverse);
    for (uint32_t c = 0; c < N; c++) pm_line(re + c, im + c, N, N, s->twr, s->twi, inverse);
}

/* mesh.rs solve + charge.rs apply: returns 0 when the mesh does not apply
 * (fewer than two nodes, distanceMax 0, no finite extent). */
static int d3_mesh(orc_d3 *s) {
    double dmin2 = s->P.distance_min * s->P.distance_min, dmax2 = s->P.distance_max * s->P.distance_max;
    if (s->n < 2 || !(dmax2 > 0.0)) return 0;
    double lx = INFINITY, ly = INFINITY, hx = -INFINITY, hy = -INFINITY;
    for (uint32_t i = 0; i < s->n; i++) {
        if (!isfinite(s->x[i]) || !isfinite(s->y[i])) continue;
        lx = fmin(lx, s->x[i]);
        ly = fmin(ly, s->y[i]);
        hx = fmax(hx, s->x[i]);
        hy = fmax(hy, s->y[i]);
    }
    if (!(lx <= hx)) return 0;
    uint32_t N = s->side;
    pm_frame f;
    if (!pm_place(lx, ly, hx, hy, N, sqrt(dmax2), &f)) return 0;
    size_t NN = (size_t)N * N;
    memset(s->gre, 0, NN * 8);
    memset(s->gim, 0, NN * 8);
    for (uint32_t i = 0; i < s->n; i++) { /* deposit.rs: cloud in cell */
        uint32_t cx, cy;
        double fx, fy;
        pm_split(&f, s->x[i], s->y[i], &cx, &cy, &fx, &fy);
        size_t at = (size_t)cy * N + cx;
        s->gre[at] += (1.0 - fx) * (1.0 - fy);
        s->gre[at + 1] += fx * (1.0 - fy);
        s->gre[at + N] += (1.0 - fx) * fy;
        s->gre[at + N + 1] += fx * fy;
    }
    /* kernel.rs sample + green */
    memset(s->kre, 0, NN * 8);
    memset(s->kim, 0, NN * 8);
    double scale = 1.0 / (double)NN;
    int reach = (int)f.reach;
    for (int dy = -reach; dy <= reach; dy++) {
        size_t row = (size_t)((dy % (int)N + (int)N) % (int)N) * N;
        for (int dx = -reach; dx <= reach; dx++) {
            double rx = (double)dx * f.h, ry = (double)dy * f.h;
            double l = rx * rx + ry * ry;
            size_t at = row + (size_t)((dx % (int)N + (int)N) % (int)N);
            if (l == 0.0 || l >= dmax2) {
                s->kre[at] = 0.0;
                s->kim[at] = 0.0;
                continue;
            }
            if (l < dmin2) l = sqrt(dmin2 * l);
            s->kre[at] = -rx / l * scale;
            s->kim[at] = -ry / l * scale;
        }
    }
    pm_fft2(s, s->kre, s->kim, 0);
    pm_fft2(s, s->gre, s->gim, 0);
    for (size_t q = 0; q < NN; q++) {
        double a = s->gre[q], b = s->gim[q], c = s->kre[q], d = s->kim[q];
        s->gre[q] = a * c - b * d;
        s->gim[q] = a * d + b * c;
    }
    pm_fft2(s, s->gre, s->gim, 1);
    double strength = s->P.charge * s->alpha;
    for (uint32_t i = 0; i < s->n; i++) { /* mesh.rs read: bilinear */
        uint32_t cx, cy;
        double fx, fy;
        pm_split(&f, s->x[i], s->y[i], &cx, &cy, &fx, &fy);
        size_t at = (size_t)cy * N + cx;
        double w[4] = {(1.0 - fx) * (1.0 - fy), fx * (1.0 - fy), (1.0 - fx) * fy, fx * fy};
        size_t cell[4] = {at, at + 1, at + N, at + N + 1};
        double ex = 0.0, ey = 0.0;
        for (int k = 0; k < 4; k++) {
            ex += s->gre[cell[k]] * w[k];
            ey += s->gim[cell[k]] * w[k];
        }
        s->dvx[i] = ex * strength;
        s->dvy[i] = ey * strength;
    }
    for (uint32_t i = 0; i < s->n; i++) {
        s->vx[i] += s->dvx[i];
        s->vy[i] += s->dvy[i];
    }
    return 1;
}

/* The mesh's field (re, im) at every node for the current positions, without
 * touching the velocities: charge * alpha left out (tests against the direct
 * law, particle_mesh/tests.rs:44-69). */
int orc_pm_field(orc_d3 *s, double *out) {
    double keep_alpha = s->alpha, keep_charge = s->P.charge;
    double *vx = (double *)malloc((size_t)(s->n ? s->n : 1) * 8), *vy = (double *)malloc((size_t)(s->n ? s->n : 1) * 8);
    memcpy(vx, s->vx, (size_t)s->n * 8);
    memcpy(vy, s->vy, (size_t)s->n * 8);
    s->alpha = 1.0;
    s->P.charge = 1.0;
    int ok = d3_mesh(s);
    for (uint32_t i = 0; i < s->n; i++) {
        out[2 * i] = ok ? s->dvx[i] : 0.0;
        out[2 * i + 1] = ok ? s->dvy[i] : 0.0;
    }
    memcpy(s->vx, vx, (size_t)s->n * 8);
    memcpy(s->vy, vy, (size_t)s->n * 8);
    free(vx);
    free(vy);
    s->alpha = keep_alpha;
    s->P.charge = keep_charge;
    return ok;
}

/* ForceSession::with_particle_mesh: the many-body pass moves onto the mesh. */
void orc_d3_use_mesh(orc_d3 *s) {
    s->mesh = 1;
    s->side = pm_side(s->n);
    size_t NN = (size_t)s->side * s->side;
    s->gre = (double *)calloc(NN, 8);
    s->gim = (double *)calloc(NN, 8);
    s->kre = (double *)calloc(NN, 8);
    s->kim = (double *)calloc(NN, 8);
    s->twr = (double *)malloc((size_t)s->side / 2 * 8);
    s->twi = (double *)malloc((size_t)s->side / 2 * 8);
    for (uint32_t k = 0; k < s->side / 2; k++) { /* fft.rs Plan::new root */
        double angle = -6.283185307179586 * (double)k / (double)s->side; /* -TAU k / side */
        s->twr[k] = cos(angle);
        s->twi[k] = sin(angle);
    }
}

/* sim.rs tick (particle_mesh.rs tick): alpha decay, link, charge, center,
 * collide, integrate. */
void orc_d3_tick(orc_d3 *s, uint32_t ticks) {
    for (uint32_t t = 0; t < ticks; t++) {
        s->alpha += (0.0 - s->alpha) * s->P.alpha_decay;
        d3_link(s);
        if (s->mesh)
            (void)d3_mesh(s);
        else
            d3_charge(s);
        d3_center(s);
        d3_collide(s);
        double decay = s->P.velocity_decay;
        for (uint32_t i = 0; i < s->n; i++) {
            s->vx[i] *= decay;
            s->x[i] += s->vx[i];
            s->vy[i] *= decay;
            s->y[i] += s->vy[i];
        }
        s->tick_no++;
    }
}

void orc_d3_positions(const orc_d3 *s, double *out) {
    for (uint32_t i = 0; i < s->n; i++) {
        out[2 * i] = s->x[i];
        out[2 * i + 1] = s->y[i];
    }
}

void orc_d3_velocities(const orc_d3 *s, double *out) {
    for (uint32_t i = 0; i < s->n; i++) {
        out[2 * i] = s->vx[i];
        out[2 * i + 1] = s->vy[i];
    }
}

double orc_d3_alpha(const orc_d3 *s) { return s->alpha; }

/* Replaces positions and velocities (n x 2 each), alpha and the tick count. */
void orc_d3_set_state(orc_d3 *s, const double *pos, const double *vel, double alpha, uint32_t tick_no) {
    for (uint32_t i = 0; i < s->n; i++) {
        s->x[i] = pos[2 * i];
        s->y[i] = pos[2 * i + 1];
        s->vx[i] = vel[2 * i];
        s->vy[i] = vel[2 * i + 1];
    }
    s->alpha = alpha;
    s->tick_no = tick_no;
}
