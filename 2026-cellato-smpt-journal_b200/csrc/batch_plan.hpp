// Work lists of the persistent batched temporal kernel (temporal_batch_kernel),
// shared by cellato_batch_create and cellato_batch_run_noalloc.
//
// Grids of one rule form a group that advances in rounds of k fused steps (k per
// rule); a grid's last round runs its remaining steps.  A group is ONE launch
// whose items -- one per (grid, round, tile) -- are claimed in list order.
// Each grid's rounds are spread evenly over the list: round r of a grid of R
// rounds sits at position (r + 1/2) * R_max / R, R_max the group's longest
// chain (ties: more rounds first).  So every stretch of the list mixes many
// grids, consecutive rounds of a grid are a whole stretch apart (a CTA rarely
// waits for the round before), and all grids finish near the end together
// instead of the longest chains running alone on an emptying device.  Round r
// of a grid reads buffer r & 1 (a, b, a, ...) and starts at step number r * k,
// whose parity the item carries.
//
// Device layout of a plan: [grid descriptors][items][one queue head per
// group][one finished-tile count per grid]; the heads and counts (the "sync"
// words) are cleared before every launch.
#ifndef CELLATO_B200_BATCH_PLAN_HPP
#define CELLATO_B200_BATCH_PLAN_HPP

#include <algorithm>
#include <numeric>
#include <vector>

#include "capi_internal.hpp"
#include "cellato_b200.h"

namespace cellato::b200::capi {

struct batch_group {
    int rule = 0, k = 8, TH = 0, HY = 0;
    int first = 0, count = 0;  // items of this group's launch
    int rounds = 0;            // longest chain of rounds
};

struct batch_plan {
    std::vector<batch_grid_desc> descs;  // per grid
    std::vector<batch_item> items;       // groups back to back
    std::vector<batch_group> groups;     // non-empty groups only
    std::vector<int> rounds;             // per grid
};

// Byte offsets of a plan's parts in one device buffer.
struct batch_layout {
    size_t items = 0, sync = 0, total = 0;  // descriptors at 0
    size_t sync_bytes = 0;                  // heads then done counts
    static size_t up(size_t v) { return (v + 255) / 256 * 256; }
    batch_layout(size_t n_grids, size_t n_items, size_t n_groups) {
        items = up(n_grids * sizeof(batch_grid_desc));
        sync = items + up(n_items * sizeof(batch_item));
        sync_bytes = (n_groups + n_grids) * sizeof(unsigned);
        total = sync + up(sync_bytes);
    }
};

// Plans the batch; max_items < 0 means no limit on the item count.
inline int plan_batch(int layout, int word_bits, const cellato_batch_grid* grids, int n_grids, const int* k_per_rule,
                      int n_k_per_rule, long long max_items, batch_plan& plan) {
    if (n_grids < 0 || (n_grids > 0 && !grids)) return fail(CELLATO_EINVAL, "bad grid array");
    if (n_k_per_rule < 0 || (n_k_per_rule > 0 && !k_per_rule)) return fail(CELLATO_EINVAL, "bad k_per_rule array");
    const int R = band_height(layout, word_bits);
    plan.descs.assign(n_grids, batch_grid_desc{});
    plan.rounds.assign(n_grids, 0);
    plan.items.clear();
    plan.groups.clear();
    std::vector<std::vector<int>> members(rule_count());
    std::vector<int> k_of(rule_count(), 8);
    for (int r = 0; r < rule_count(); ++r) {
        const int k = (k_per_rule && r < n_k_per_rule) ? k_per_rule[r] : 0;
        if (k < 0 || k > 32) return fail(CELLATO_EINVAL, "k for rule %d must be in 1..32 (0 = 8), got %d", r, k);
        k_of[r] = k > 0 ? k : 8;
    }
    for (int i = 0; i < n_grids; ++i) {
        const cellato_batch_grid& g = grids[i];
        const rule_ops* ops = ops_of(g.rule);
        if (!ops) return fail(CELLATO_EINVAL, "grid %d: unknown rule id %d", i, g.rule);
        if (g.steps < 0) return fail(CELLATO_EINVAL, "grid %d: negative step count", i);
        if (int rc = check_dims(layout, word_bits, g.x_cells, g.y_cells)) return rc;
        plane_set pa, pb;
        if (int rc = make_sets(ops, g.planes_a, g.planes_b, pa, pb)) return rc;
        plan.descs[i].p[0] = pa;
        plan.descs[i].p[1] = pb;
        plan.descs[i].Xw = g.x_cells / 32;
        plan.descs[i].Y = g.y_cells;
        plan.rounds[i] = (g.steps + k_of[g.rule] - 1) / k_of[g.rule];
        members[g.rule].push_back(i);
    }
    for (int rule = 0; rule < rule_count(); ++rule) {
        if (members[rule].empty()) continue;
        const rule_ops* ops = ops_of(rule);
        batch_group gp;
        gp.rule = rule;
        gp.k = k_of[rule];
        gp.TH = default_tile_rows(ops, R, gp.k, ops->batch_words_per_lane);
        gp.HY = (gp.k + R - 1) / R * R;
        const int effW = 32 * ops->batch_words_per_lane - 2, effH = gp.TH - 2 * gp.HY;
        if (effH <= 0)
            return fail(CELLATO_EINVAL, "rule %d: a %d-row tile leaves no interior for k=%d", rule, gp.TH, gp.k);
        std::vector<int>& m = members[rule];
        for (int i : m) {
            const int tx = (plan.descs[i].Xw + effW - 1) / effW, ty = (plan.descs[i].Y + effH - 1) / effH;
            plan.descs[i].tiles = tx * ty;
            gp.rounds = std::max(gp.rounds, plan.rounds[i]);
        }
        // (position numerator, grid, round); position = (2r + 1) * R_max / (2 R)
        struct slot_t {
            long long num, den;
            int grid, round;
        };
        std::vector<slot_t> order;
        for (int i : m)
            for (int r = 0; r < plan.rounds[i]; ++r)
                order.push_back(slot_t{(2LL * r + 1) * gp.rounds, 2LL * plan.rounds[i], i, r});
        std::stable_sort(order.begin(), order.end(), [&](const slot_t& a, const slot_t& b) {
            const long long l = a.num * b.den, r = b.num * a.den;
            if (l != r) return l < r;
            return plan.rounds[a.grid] > plan.rounds[b.grid];
        });
        gp.first = (int)plan.items.size();
        for (const slot_t& o : order) {
            const int i = o.grid, r = o.round;
            const int steps = std::min(gp.k, grids[i].steps - r * gp.k);
            const int flags = steps | ((r & 1) ? BATCH_FLIP_BUFFER : 0) |
                              (((long long)r * gp.k) & 1 ? BATCH_FLIP_TIME : 0) | (r << BATCH_ROUND_SHIFT);
            const int tx = (plan.descs[i].Xw + effW - 1) / effW, ty = plan.descs[i].tiles / tx;
            if (max_items >= 0 && (long long)plan.items.size() + tx * ty > max_items)
                return fail(CELLATO_EINVAL,
                            "the batch needs more than %lld work items (tiles x rounds), the no-allocation limit",
                            max_items);
            for (int y = 0; y < ty; ++y)
                for (int x = 0; x < tx; ++x) plan.items.push_back(batch_item{i, x, y, flags});
        }
        gp.count = (int)plan.items.size() - gp.first;
        if (gp.count > 0) plan.groups.push_back(gp);
    }
    return CELLATO_OK;
}

// Enqueues one persistent launch per group on `s` (or on the group's own
// stream), each with the resident CTAs the device holds (sms x CTAs per SM, at
// most one per item).  The sync words must be zero (stream-ordered) when the
// launches run, and each group's kernel attributes must have been set
// (rule_ops::prepare_batch, outside any stream capture).
inline int launch_plan(const batch_plan& plan, int internal, const batch_grid_desc* d_descs,
                       const batch_item* d_items, unsigned* d_sync, int sms, cudaStream_t s, int* launches = nullptr,
                       const std::vector<cudaStream_t>* per_group_streams = nullptr) {
    const int n_groups = (int)plan.groups.size();
    unsigned* d_done = d_sync + n_groups;
    for (int g = 0; g < n_groups; ++g) {
        const batch_group& gp = plan.groups[g];
        const rule_ops* ops = ops_of(gp.rule);
        const int per_sm = ops->batch_blocks_per_sm(internal, gp.TH);
        const int ctas = std::max(1, std::min(gp.count, per_sm * sms));
        cudaStream_t st = per_group_streams ? (*per_group_streams)[g] : s;
        const cudaError_t e = ops->temporal_batch(internal, d_descs, d_items + gp.first, gp.count, 0, 0, gp.TH, gp.HY,
                                                  d_sync + g, d_done, ctas, st);
        if (e != cudaSuccess) return cuda_fail(e, "batched temporal launch");
        if (launches) ++*launches;
    }
    return CELLATO_OK;
}

}  // namespace cellato::b200::capi

#endif  // CELLATO_B200_BATCH_PLAN_HPP
