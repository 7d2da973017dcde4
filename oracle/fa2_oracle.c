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

static void cell_push(ttree *t, const double *b0, const double *b1, uint32_t start) {
    if (t->ncells == t->capcells) {
        t->capcells = t->capcells ? t->capcells * 2 : 1024;
        t->cells = (tcell *)realloc(t->cells, t->capcells * sizeof(tcell));
    }
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
        cell_push(t, v.b0, v.b1, start);
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
