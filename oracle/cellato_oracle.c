/*
 * Test infrastructure only -- the oracle.  A plain-C restatement of the
 * reference's CPU "standard" evaluator path for the ten automata, plus the
 * bit-plane packing rules and the 4x4 tile checksum.  Only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it, and only
 * as the checker; the product never links it.
 *
 * Cells are uint8 *dictionary indices*: the integer a bit-plane layout
 * encodes, bit i of the index living in plane i
 * (include/memory/state_dictionary.hpp:24-45, include/memory/bit_planes_grid.hpp:255-263).
 * Each rule below is the reference rule restated over indices; the index order
 * is the order of the automaton's state_dictionary (src/<a>/config.hpp).
 *
 * Grid semantics (reference file:line):
 *   - torus wrap on both axes: include/memory/interface.hpp:28-33
 *   - one step = evaluate every cell of `cur` into `nxt`, time_step = step index:
 *     include/traversers/cpu/simple.hpp:60-85
 *   - count_neighbors Moore order/offsets: include/evaluators/standard.hpp:160-173
 *   - von Neumann offsets: include/evaluators/standard.hpp:243-252
 *   - Margolus block and 180-degree neighbour: include/evaluators/standard.hpp:175-241
 *   - alternate_algorithms by time_step parity: include/evaluators/standard.hpp:150-158
 */
#define _GNU_SOURCE
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORACLE_RULES 10

enum {
    R_GOL = 0, R_FIRE, R_WIRE, R_EXCITABLE, R_BRIAN, R_MAZE, R_CYCLIC, R_FLUID, R_CRITTERS, R_TRAFFIC
};

static const char* k_names[ORACLE_RULES] = {
    "game-of-life", "forest-fire", "wire", "excitable", "brian",
    "maze", "cyclic", "fluid", "critters", "traffic"};

/* needed_bits = log2(n-1)+1 (state_dictionary.hpp:22) or the int dictionary width (:48-70). */
static const int k_planes[ORACLE_RULES] = {1, 2, 2, 3, 2, 1, 5, 4, 1, 2};
static const int k_states[ORACLE_RULES] = {2, 4, 4, 8, 3, 2, 32, 16, 2, 3};

const char* oracle_rule_name(int rule) { return (rule >= 0 && rule < ORACLE_RULES) ? k_names[rule] : 0; }
int oracle_rule_count(void) { return ORACLE_RULES; }
int oracle_planes(int rule) { return (rule >= 0 && rule < ORACLE_RULES) ? k_planes[rule] : -1; }
int oracle_states(int rule) { return (rule >= 0 && rule < ORACLE_RULES) ? k_states[rule] : -1; }
int oracle_rule_from_name(const char* s) {
    if (!s) return -1;
    for (int r = 0; r < ORACLE_RULES; ++r)
        if (strcmp(s, k_names[r]) == 0) return r;
    if (strcmp(s, "fire") == 0) return R_FIRE; /* main.cpp:61 accepts both */
    return -1;
}

/* Index -> enum value.  Only forest-fire's dictionary order differs from its
 * enum order: dictionary {empty, tree, fire, ash} (src/fire/config.hpp:22-24),
 * enum {empty=0, tree=1, ash=2, fire=3} (src/fire/algorithm.hpp:9-14). */
int oracle_state_value(int rule, int index) {
    if (rule == R_FIRE) {
        static const int v[4] = {0, 1, 3, 2};
        return (index >= 0 && index < 4) ? v[index] : -1;
    }
    return index;
}

typedef struct {
    const uint8_t* g;
    int X, Y;
} grid_t;

static inline uint8_t at(const grid_t* g, int x, int y) {
    /* interface.hpp:28-33: (x + X) % X; every offset used here is within +-1,
     * so the wrap is a single conditional add or subtract. */
    int xr = x < 0 ? x + g->X : (x >= g->X ? x - g->X : x);
    int yr = y < 0 ? y + g->Y : (y >= g->Y ? y - g->Y : y);
    return g->g[(size_t)yr * g->X + xr];
}

static inline int moore_count(const grid_t* g, int x, int y, uint8_t v) {
    static const int dx[8] = {-1, 0, 1, -1, 1, -1, 0, 1};
    static const int dy[8] = {-1, -1, -1, 0, 0, 1, 1, 1};
    int c = 0;
    for (int i = 0; i < 8; ++i) c += at(g, x + dx[i], y + dy[i]) == v;
    return c;
}

static inline int von_neumann_count(const grid_t* g, int x, int y, uint8_t v) {
    return (at(g, x, y + 1) == v) + (at(g, x, y - 1) == v) + (at(g, x + 1, y) == v) + (at(g, x - 1, y) == v);
}

/* src/game_of_life/algorithm.hpp:35-49; dictionary {dead, alive}. */
static uint8_t rule_gol(const grid_t* g, int x, int y, int t) {
    (void)t;
    int c = moore_count(g, x, y, 1);
    if (at(g, x, y) == 1) return (c == 2 || c == 3) ? 1 : 0;
    return c == 3 ? 1 : 0;
}

/* src/fire/algorithm.hpp:39-57; dictionary {empty=0, tree=1, fire=2, ash=3}. */
static uint8_t rule_fire(const grid_t* g, int x, int y, int t) {
    (void)t;
    uint8_t s = at(g, x, y);
    if (s == 2) return 3;
    if (s == 3) return von_neumann_count(g, x, y, 2) > 0 ? 3 : 0;
    if (s == 1) return von_neumann_count(g, x, y, 2) > 0 ? 2 : 1;
    return 0;
}

/* src/wire/algorithm.hpp:48-59; dictionary {empty, head, tail, conductor}. */
static uint8_t rule_wire(const grid_t* g, int x, int y, int t) {
    (void)t;
    uint8_t s = at(g, x, y);
    if (s == 1) return 2;
    if (s == 2) return 3;
    if (s == 3) {
        int c = moore_count(g, x, y, 1);
        return (c == 1 || c == 2) ? 1 : 3;
    }
    return 0;
}

/* src/excitable/algorithm.hpp:57-71; dictionary {quiescent, excited, r1..r6}. */
static uint8_t rule_excitable(const grid_t* g, int x, int y, int t) {
    (void)t;
    uint8_t s = at(g, x, y);
    if (s == 0) return moore_count(g, x, y, 1) > 0 ? 1 : 0;
    if (s <= 6) return (uint8_t)(s + 1);
    return 0;
}

/* src/brian/algorithm.hpp:31-44; dictionary {dead, dying, alive}. */
static uint8_t rule_brian(const grid_t* g, int x, int y, int t) {
    (void)t;
    uint8_t s = at(g, x, y);
    if (s == 0) return moore_count(g, x, y, 2) == 2 ? 2 : 0;
    if (s == 2) return 1;
    return 0;
}

/* src/maze/algorithm.hpp:29-35; dictionary {empty, wall}. */
static uint8_t rule_maze(const grid_t* g, int x, int y, int t) {
    (void)t;
    int c = moore_count(g, x, y, 1);
    if (c == 3) return 1;
    if (at(g, x, y) == 1 && c < 6) return 1;
    return 0;
}

/* src/cyclic/algorithm.hpp:11-23; int dictionary of 5 bits. */
static uint8_t rule_cyclic(const grid_t* g, int x, int y, int t) {
    (void)t;
    uint8_t s = at(g, x, y);
    uint8_t nx = (uint8_t)((s + 1) % 32);
    return moore_count(g, x, y, nx) > 0 ? nx : s;
}

/* src/fluid/algorithm.hpp:11-60; int dictionary of 4 bits,
 * TOP=1, BOTTOM=2, LEFT=4, RIGHT=8. */
static uint8_t rule_fluid(const grid_t* g, int x, int y, int t) {
    (void)t;
    uint8_t up = at(g, x, y - 1), down = at(g, x, y + 1);
    uint8_t left = at(g, x - 1, y), right = at(g, x + 1, y);
    int in_top = (up & 1) != 0, in_bottom = (down & 2) != 0;
    int in_left = (left & 4) != 0, in_right = (right & 8) != 0;
    int vcoll = in_top & in_bottom, hcoll = in_left & in_right;
    int cvi = (up & 1) | (down & 2);
    int chi = (left & 4) | (right & 8);
    int just_v = vcoll & (chi == 0);
    int just_h = hcoll & (cvi == 0);
    int vres = just_v ? (4 | 8) : cvi;
    int hres = just_h ? (1 | 2) : chi;
    return (uint8_t)(vres | hres);
}

/* Margolus block offsets, include/evaluators/standard.hpp:175-205 (count) and
 * :207-241 (180-degree neighbour).  Parity of the step, x and y selects which
 * of the two partners along each axis belongs to the block. */
static inline int margolus_dx(int x, int t) { return ((t & 1) == 0) ? ((x & 1) == 0 ? 1 : -1) : ((x & 1) == 0 ? -1 : 1); }
static inline int margolus_dy(int y, int t) { return ((t & 1) == 0) ? ((y & 1) == 0 ? 1 : -1) : ((y & 1) == 0 ? -1 : 1); }

/* src/critters/algorithm.hpp:16-31; dictionary {dead, alive}. */
static uint8_t rule_critters(const grid_t* g, int x, int y, int t) {
    int dx = margolus_dx(x, t), dy = margolus_dy(y, t);
    uint8_t s = at(g, x, y);
    int c = (s == 1) + (at(g, x + dx, y) == 1) + (at(g, x, y + dy) == 1) + (at(g, x + dx, y + dy) == 1);
    if (c == 3) return at(g, x + dx, y + dy) == 1 ? 0 : 1;
    if (c == 2) return s;
    return s == 1 ? 0 : 1;
}

/* src/traffic/algorithm.hpp:15-61; dictionary {empty, red_car, blue_car}.
 * Even steps: red moves right; odd steps: blue moves down. */
static uint8_t rule_traffic(const grid_t* g, int x, int y, int t) {
    uint8_t s = at(g, x, y);
    if ((t & 1) == 0) {
        if (s == 1) return at(g, x + 1, y) == 0 ? 0 : 1;
        if (s == 0) return at(g, x - 1, y) == 1 ? 1 : 0;
        return 2;
    }
    if (s == 2) return at(g, x, y + 1) == 0 ? 0 : 2;
    if (s == 0) return at(g, x, y - 1) == 2 ? 2 : 0;
    return 1;
}

typedef uint8_t (*rule_fn)(const grid_t*, int, int, int);
static const rule_fn k_rules[ORACLE_RULES] = {rule_gol, rule_fire, rule_wire, rule_excitable, rule_brian,
                                              rule_maze, rule_cyclic, rule_fluid, rule_critters, rule_traffic};

typedef struct {
    int rule, X, Y, y0, y1, t0, steps, nthreads;
    uint8_t *a, *b;
    pthread_barrier_t* bar;
} job_t;

static void* worker(void* p) {
    job_t* j = (job_t*)p;
    rule_fn f = k_rules[j->rule];
    uint8_t* cur = j->a;
    uint8_t* nxt = j->b;
    for (int s = 0; s < j->steps; ++s) {
        grid_t g = {cur, j->X, j->Y};
        int t = j->t0 + s;
        for (int y = j->y0; y < j->y1; ++y)
            for (int x = 0; x < j->X; ++x) nxt[(size_t)y * j->X + x] = f(&g, x, y, t);
        uint8_t* tmp = cur;
        cur = nxt;
        nxt = tmp;
        if (j->nthreads > 1) pthread_barrier_wait(j->bar);
    }
    return 0;
}

/* Run `steps` steps starting at global step index t0 (parity of t0 matters for
 * critters and traffic).  `in` and `out` may alias.  Returns 0 on success. */
int oracle_run(int rule, const uint8_t* in, uint8_t* out, int X, int Y, int t0, int steps, int threads) {
    if (rule < 0 || rule >= ORACLE_RULES || X <= 0 || Y <= 0 || steps < 0) return -1;
    size_t n = (size_t)X * Y;
    uint8_t* a = (uint8_t*)malloc(n);
    uint8_t* b = (uint8_t*)malloc(n);
    if (!a || !b) {
        free(a);
        free(b);
        return -3;
    }
    memcpy(a, in, n);
    memcpy(b, in, n);
    if (threads < 1) threads = 1;
    if (threads > Y) threads = Y;
    pthread_barrier_t bar;
    if (threads > 1) pthread_barrier_init(&bar, 0, (unsigned)threads);
    job_t* jobs = (job_t*)calloc((size_t)threads, sizeof(job_t));
    pthread_t* th = (pthread_t*)calloc((size_t)threads, sizeof(pthread_t));
    for (int i = 0; i < threads; ++i) {
        jobs[i] = (job_t){rule, X, Y, (int)((long long)Y * i / threads), (int)((long long)Y * (i + 1) / threads),
                          t0, steps, threads, a, b, &bar};
        if (i > 0) pthread_create(&th[i], 0, worker, &jobs[i]);
    }
    worker(&jobs[0]);
    for (int i = 1; i < threads; ++i) pthread_join(th[i], 0);
    if (threads > 1) pthread_barrier_destroy(&bar);
    memcpy(out, (steps % 2 == 0) ? a : b, n);
    free(jobs);
    free(th);
    free(a);
    free(b);
    return 0;
}

/* ---- layouts (the byte formats the GPU path must read and write) ----
 * Linear bit planes, include/memory/bit_planes_grid.hpp:234-270: plane p is
 * Y rows of X/W words; word (wx, y) bit i holds bit p of cell (wx*W + i, y)
 * -- least significant bit = leftmost cell.
 * Tiled bit planes, include/memory/tiled_bit_planes_grid.hpp:243-288: a word
 * covers 8 cells across and W/8 rows down; bit (yb*8 + xb) holds cell
 * (tx*8 + xb, ty*(W/8) + yb); words are stored row-major by tile.
 * Both are written as little-endian words; `planes` is nb planes laid back to
 * back, each X*Y/8 bytes. */
static inline size_t bit_pos_linear(int x, int y, int X, int W) {
    size_t word = (size_t)y * (X / W) + (size_t)(x / W);
    return word * W + (x % W);
}

static inline size_t bit_pos_tiled(int x, int y, int X, int W) {
    int R = W / 8;
    size_t word = (size_t)(y / R) * (X / 8) + (size_t)(x / 8);
    return word * W + (size_t)((y % R) * 8 + (x % 8));
}

int oracle_pack(int layout, int W, int nb, const uint8_t* cells, int X, int Y, uint8_t* planes) {
    if ((W != 32 && W != 64) || nb < 1 || nb > 8) return -1;
    if (layout == 0 && X % W != 0) return -1;
    if (layout == 1 && (X % 8 != 0 || Y % (W / 8) != 0)) return -1;
    size_t plane_bytes = (size_t)X * Y / 8;
    memset(planes, 0, plane_bytes * nb);
    for (int y = 0; y < Y; ++y)
        for (int x = 0; x < X; ++x) {
            size_t bp = layout == 0 ? bit_pos_linear(x, y, X, W) : bit_pos_tiled(x, y, X, W);
            uint8_t v = cells[(size_t)y * X + x];
            for (int p = 0; p < nb; ++p)
                if ((v >> p) & 1) planes[p * plane_bytes + bp / 8] |= (uint8_t)(1u << (bp % 8));
        }
    return 0;
}

int oracle_unpack(int layout, int W, int nb, const uint8_t* planes, int X, int Y, uint8_t* cells) {
    if ((W != 32 && W != 64) || nb < 1 || nb > 8) return -1;
    if (layout == 0 && X % W != 0) return -1;
    if (layout == 1 && (X % 8 != 0 || Y % (W / 8) != 0)) return -1;
    size_t plane_bytes = (size_t)X * Y / 8;
    for (int y = 0; y < Y; ++y)
        for (int x = 0; x < X; ++x) {
            size_t bp = layout == 0 ? bit_pos_linear(x, y, X, W) : bit_pos_tiled(x, y, X, W);
            uint8_t v = 0;
            for (int p = 0; p < nb; ++p) v |= (uint8_t)(((planes[p * plane_bytes + bp / 8] >> (bp % 8)) & 1) << p);
            cells[(size_t)y * X + x] = v;
        }
    return 0;
}

/* 4x4 tile sums of the state *values* (standard_grid.hpp:179-213): tile sides
 * are ceil(X/4) x ceil(Y/4); sums are written to out[16] in row-major tile order. */
int oracle_checksum(int rule, const uint8_t* cells, int X, int Y, uint64_t* out) {
    if (rule < 0 || rule >= ORACLE_RULES) return -1;
    const int dims = 4;
    int tw = (X + dims - 1) / dims, th = (Y + dims - 1) / dims;
    int lut[256];
    for (int i = 0; i < 256; ++i) lut[i] = oracle_state_value(rule, i);
    for (int ty = 0; ty < dims; ++ty)
        for (int tx = 0; tx < dims; ++tx) {
            int sx = tx * tw, sy = ty * th;
            int ex = sx + tw < X ? sx + tw : X, ey = sy + th < Y ? sy + th : Y;
            uint64_t s = 0;
            for (int y = sy; y < ey; ++y)
                for (int x = sx; x < ex; ++x) s += (uint64_t)lut[cells[(size_t)y * X + x]];
            out[ty * dims + tx] = s;
        }
    return 0;
}
