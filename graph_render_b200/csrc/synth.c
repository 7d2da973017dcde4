/*
 * Seeded synthetic graphs and start positions for the workloads the engine is
 * measured on: stochastic block models, Barabasi-Albert preferential
 * attachment, a power-law configuration model, a 2D grid with rewiring, and
 * uniform boxes of start positions. Host code; every generator is a pure
 * function of its arguments and seed (SplitMix64 stream).
 *
 * Edges come out as raw (src, dst) pairs; duplicates and self-loops are left in
 * for the engine's simple-graph pass to drop, as a topology's would be
 * (crates/graph-core/src/layout/force/mod.rs:101-120).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct { uint64_t s; } sm64;

static uint64_t sm_next(sm64 *r) {
    uint64_t z = (r->s += 0x9e3779b97f4a7c15ULL);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

/* uniform in [0, 1) with 53 bits */
static double sm_unit(sm64 *r) { return (double)(sm_next(r) >> 11) * (1.0 / 9007199254740992.0); }

static uint64_t sm_below(sm64 *r, uint64_t n) { return n ? sm_next(r) % n : 0; }

static double sm_normal(sm64 *r) {
    double u = sm_unit(r), v = sm_unit(r);
    if (u < 1e-300) u = 1e-300;
    return sqrt(-2.0 * log(u)) * cos(6.283185307179586 * v);
}

/* Edge sink with a hard capacity; counts past it so the caller can size. */
typedef struct {
    uint32_t *src, *dst;
    int64_t cap, m;
} sink;

static void put(sink *k, uint32_t a, uint32_t b) {
    if (k->m < k->cap) {
        k->src[k->m] = a;
        k->dst[k->m] = b;
    }
    k->m++;
}

/* Geometric skip: gap to the next success of a Bernoulli(p) sequence. */
static uint64_t geo_skip(sm64 *r, double lp) {
    double u = sm_unit(r);
    if (u < 1e-300) u = 1e-300;
    return (uint64_t)floor(log(u) / lp);
}

/* Stochastic block model: blocks of sizes[b], edge probability p_in inside a
 * block and p_out between blocks, sampled by geometric skipping over the pair
 * index so the cost is the number of edges, not of pairs. */
int64_t syn_sbm(uint32_t nblocks, const uint32_t *sizes, double p_in, double p_out, uint64_t seed,
                uint32_t *src, uint32_t *dst, int64_t cap) {
    sm64 r = {seed};
    sink k = {src, dst, cap, 0};
    uint32_t *off = (uint32_t *)malloc((nblocks + 1) * sizeof(uint32_t));
    off[0] = 0;
    for (uint32_t b = 0; b < nblocks; b++) off[b + 1] = off[b] + sizes[b];
    for (uint32_t a = 0; a < nblocks; a++)
        for (uint32_t b = a; b < nblocks; b++) {
            double p = a == b ? p_in : p_out;
            if (p <= 0.0) continue;
            uint64_t sa = sizes[a], sb = sizes[b];
            uint64_t npairs = a == b ? sa * (sa - 1) / 2 : sa * sb;
            double lp = log1p(-fmin(p, 1.0 - 1e-16));
            uint64_t t = p >= 1.0 ? 0 : geo_skip(&r, lp);
            while (t < npairs) {
                uint32_t i, j;
                if (a == b) {
                    /* t -> (i, j), i > j, row i holds i pairs */
                    uint64_t ii = (uint64_t)floor((1.0 + sqrt(1.0 + 8.0 * (double)t)) / 2.0);
                    while (ii * (ii - 1) / 2 > t) ii--;
                    while ((ii + 1) * ii / 2 <= t) ii++;
                    i = (uint32_t)ii;
                    j = (uint32_t)(t - ii * (ii - 1) / 2);
                    put(&k, off[a] + i, off[a] + j);
                } else {
                    i = (uint32_t)(t / sb);
                    j = (uint32_t)(t % sb);
                    put(&k, off[a] + i, off[b] + j);
                }
                t += 1 + (p >= 1.0 ? 0 : geo_skip(&r, lp));
            }
        }
    free(off);
    return k.m;
}

/* Barabasi-Albert: a star over the first m+1 nodes, then each new node links
 * to m distinct earlier nodes drawn with probability proportional to degree
 * (a uniform pick from the list of edge endpoints). */
int64_t syn_ba(uint32_t n, uint32_t m, uint64_t seed, uint32_t *src, uint32_t *dst, int64_t cap) {
    sm64 r = {seed};
    sink k = {src, dst, cap, 0};
    if (n < 2 || m < 1) return 0;
    if (m >= n) m = n - 1;
    uint64_t ecap = 2 * ((uint64_t)m * n + 1);
    uint32_t *ends = (uint32_t *)malloc(ecap * sizeof(uint32_t));
    uint64_t ne = 0;
    for (uint32_t i = 1; i <= m; i++) {
        put(&k, i, 0);
        ends[ne++] = i;
        ends[ne++] = 0;
    }
    uint32_t *pick = (uint32_t *)malloc(m * sizeof(uint32_t));
    for (uint32_t v = m + 1; v < n; v++) {
        uint32_t got = 0;
        while (got < m) {
            uint32_t t = ends[sm_below(&r, ne)];
            int dup = 0;
            for (uint32_t q = 0; q < got; q++)
                if (pick[q] == t) dup = 1;
            if (!dup) pick[got++] = t;
        }
        for (uint32_t q = 0; q < m; q++) {
            put(&k, v, pick[q]);
            ends[ne++] = v;
            ends[ne++] = pick[q];
        }
    }
    free(pick);
    free(ends);
    return k.m;
}

/* Configuration model with power-law degrees: k = max(kmin, floor(x)), x Pareto
 * with exponent `alpha` and scale `xmin` (kmin = 2 and xmin = 2.83 give a mean
 * near 8 at alpha 2.5), capped at n - 1; stubs shuffled and paired. */
int64_t syn_config_powerlaw(uint32_t n, double alpha, uint32_t kmin, double xmin, uint64_t seed,
                            uint32_t *src, uint32_t *dst, int64_t cap) {
    sm64 r = {seed};
    sink k = {src, dst, cap, 0};
    uint32_t *deg = (uint32_t *)malloc((size_t)(n ? n : 1) * sizeof(uint32_t));
    uint64_t total = 0;
    for (uint32_t i = 0; i < n; i++) {
        double u = sm_unit(&r);
        if (u < 1e-300) u = 1e-300;
        double x = xmin * pow(u, -1.0 / (alpha - 1.0));
        double d = floor(x);
        if (d < kmin) d = kmin;
        if (d > n - 1) d = n - 1;
        deg[i] = (uint32_t)d;
        total += deg[i];
    }
    if (total & 1) {
        deg[0]++;
        total++;
    }
    uint32_t *stubs = (uint32_t *)malloc((size_t)(total ? total : 1) * sizeof(uint32_t));
    uint64_t q = 0;
    for (uint32_t i = 0; i < n; i++)
        for (uint32_t d = 0; d < deg[i]; d++) stubs[q++] = i;
    for (uint64_t i = total; i > 1; i--) {
        uint64_t j = sm_below(&r, i);
        uint32_t t = stubs[i - 1];
        stubs[i - 1] = stubs[j];
        stubs[j] = t;
    }
    for (uint64_t i = 0; i + 1 < total; i += 2) put(&k, stubs[i], stubs[i + 1]);
    free(stubs);
    free(deg);
    return k.m;
}

/* A side x side grid (node = row * side + col, the last row possibly short to
 * hold exactly n nodes), right and down links, then each link rewired with
 * probability `rewire` to a uniform random node. */
int64_t syn_grid(uint32_t n, double rewire, uint64_t seed, uint32_t *src, uint32_t *dst, int64_t cap) {
    sm64 r = {seed};
    sink k = {src, dst, cap, 0};
    uint32_t side = (uint32_t)ceil(sqrt((double)n));
    if (side == 0) return 0;
    for (uint32_t v = 0; v < n; v++) {
        uint32_t row = v / side, c = v % side;
        uint32_t nb[2];
        int cnt = 0;
        if (c + 1 < side && v + 1 < n) nb[cnt++] = v + 1;
        if (v + side < n) nb[cnt++] = v + side;
        (void)row;
        for (int q = 0; q < cnt; q++) {
            uint32_t t = nb[q];
            if (sm_unit(&r) < rewire) t = (uint32_t)sm_below(&r, n);
            put(&k, v, t);
        }
    }
    return k.m;
}

/* n x dim start positions uniform in [lo, hi)^dim, row-major. */
void syn_uniform(uint32_t n, uint32_t dim, double lo, double hi, uint64_t seed, float *out) {
    sm64 r = {seed};
    for (uint64_t i = 0; i < (uint64_t)n * dim; i++) out[i] = (float)(lo + (hi - lo) * sm_unit(&r));
}

/* Lognormal(mu, sigma) edge weights. */
void syn_lognormal(uint64_t m, double mu, double sigma, uint64_t seed, double *out) {
    sm64 r = {seed};
    for (uint64_t e = 0; e < m; e++) out[e] = exp(mu + sigma * sm_normal(&r));
}

/* Uniform integers in [0, n) (stress-pair sampling and the like). */
void syn_randint(uint64_t count, uint32_t n, uint64_t seed, uint32_t *out) {
    sm64 r = {seed};
    for (uint64_t i = 0; i < count; i++) out[i] = (uint32_t)sm_below(&r, n);
}

/* Uniform doubles in [0, 1). */
void syn_unit(uint64_t count, uint64_t seed, double *out) {
    sm64 r = {seed};
    for (uint64_t i = 0; i < count; i++) out[i] = sm_unit(&r);
}

/* The reference's benchmark model (crates/graph-core/src/synthetic.rs:92-170,
 * the graph its `tick` and snapshot benches run on): one mulberry32 stream from
 * 0x051042, read first by the node records (an icon roll and, below 0.8, a table
 * pick), then by preferential attachment (node i to floor(u v i), a second such
 * edge with probability 1/2) and floor(0.05 n) uniform extra pairs; every edge
 * that is not a self-edge draws its strength 0.4 + 0.4 u. Returns the edge
 * count; writes at most cap edges. */
static double mb32_unit(uint32_t *s) {
    *s += 0x6D2B79F5u;
    uint32_t a = *s;
    uint32_t t = (a ^ (a >> 15)) * (1u | a);
    t = (t + ((t ^ (t >> 7)) * (61u | t))) ^ t;
    return (double)(t ^ (t >> 14)) / 4294967296.0;
}

int64_t syn_gate(uint32_t count, uint32_t *src, uint32_t *dst, double *strength, int64_t cap) {
    uint32_t s = 0x051042u;
    for (uint32_t i = 0; i < count; i++) {
        const double roll = mb32_unit(&s);
        if (roll < 0.8) (void)mb32_unit(&s); /* the emoji (12) or icon (4) pick */
    }
    int64_t m = 0;
    for (uint32_t pass = 0; pass < 2; pass++) {
        const uint32_t rounds = pass == 0 ? (count ? count - 1 : 0) : (uint32_t)floor((double)count * 0.05);
        for (uint32_t r = 0; r < rounds; r++) {
            for (int second = 0; second < 2; second++) {
                uint32_t a, b;
                if (pass == 0) {
                    const uint32_t i = r + 1;
                    if (second && !(mb32_unit(&s) < 0.5)) break;
                    const double u = mb32_unit(&s), v = mb32_unit(&s);
                    a = i;
                    b = (uint32_t)floor(u * v * (double)i);
                } else {
                    if (second) break;
                    a = (uint32_t)floor(mb32_unit(&s) * (double)count);
                    b = (uint32_t)floor(mb32_unit(&s) * (double)count);
                }
                if (a == b) continue;
                const double st = 0.4 + mb32_unit(&s) * 0.4;
                if (m < cap) {
                    src[m] = a;
                    dst[m] = b;
                    strength[m] = st;
                }
                m++;
            }
        }
    }
    return m;
}
