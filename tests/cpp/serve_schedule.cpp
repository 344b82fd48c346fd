// Host test of the server's scheduling policy (csrc/serve_schedule.hpp).
// Random request streams are submitted while iterations run; after every
// admission and plan the invariants are checked:
//   * admission is strict FIFO in submission order and the resident bytes stay
//     within the cap (a request larger than the cap only when it is alone);
//   * the tiles of the active requests stay within the budget, or a single
//     request is active;
//   * each request's rounds, concatenated over iterations, cover exactly its
//     steps, read the buffers alternately starting with a, carry the parity of
//     their first step number, and never exceed k steps;
//   * every request finishes exactly once, with the final buffer = parity of
//     its round count;
//   * cancelling a request at any stage (preemption) removes it from the
//     queues and its bytes from the resident total.
// Prints "ok" and exits 0 on success; prints the failed check and exits 1.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <random>
#include <vector>

#include "serve_schedule.hpp"

using namespace cellato::b200::serve;

// rule ids drawn by the scenarios: the ten built-in ones and three registered
// ones; the last two have no k entry (the scheduler's default applies)
constexpr int RULES = 13;

#define CHECK(c, ...)                                   \
    do {                                                \
        if (!(c)) {                                     \
            std::printf("FAILED %s: ", #c);             \
            std::printf(__VA_ARGS__);                   \
            std::printf("\n");                          \
            std::exit(1);                               \
        }                                               \
    } while (0)

struct truth {
    int rule, steps, k;
    long long bytes;
    int tiles;
    bool keep;
    int t0 = 0;
    int done = 0, cur = 0, rounds = 0;
    bool finished = false, admitted = false;
};

int scenario(unsigned seed, long long cap, long long budget, int chunk_rounds) {
    std::mt19937 rng(seed);
    limits lim;
    lim.cap_bytes = cap;
    lim.tile_budget = budget;
    lim.chunk_rounds = chunk_rounds;
    lim.k.assign(RULES - 2, 0);
    for (int r = 0; r < RULES - 2; ++r) lim.k[r] = 1 + (int)(rng() % 20);
    scheduler sch(lim);
    std::map<long long, truth> t;
    std::vector<long long> submitted;
    size_t next_admit = 0;  // index into submitted: FIFO admission order
    int to_submit = 300, finished = 0;
    for (int it = 0; it < 100000 && finished < 300; ++it) {
        // a burst of arrivals
        const int burst = (int)(rng() % 5);
        for (int b = 0; b < burst && to_submit > 0; ++b, --to_submit) {
            truth q;
            q.rule = (int)(rng() % RULES);
            q.steps = (rng() % 10 == 0) ? 0 : 1 + (int)(rng() % 300);
            q.k = lim.k_of(q.rule);
            q.bytes = 1 + (long long)(rng() % (unsigned)(cap / 3 + 1));
            if (rng() % 50 == 0) q.bytes = cap + 5;  // larger than the cap
            q.tiles = 1 + (int)(rng() % 40);
            q.keep = rng() % 4 == 0;
            q.t0 = (int)(rng() % 4);
            const long long id = sch.submit(q.rule, 64, 64, q.steps, q.bytes, q.tiles, q.keep, q.t0);
            t[id] = q;
            submitted.push_back(id);
        }
        // now and then a live request is cancelled (preempted)
        if (rng() % 8 == 0) {
            std::vector<long long> live;
            for (auto& [id, x] : t)
                if (!x.finished) live.push_back(id);
            if (!live.empty()) {
                const long long id = live[rng() % live.size()];
                truth& x = t[id];
                const long long bytes = sch.resident_bytes();
                const int ph = sch.cancel(id);
                CHECK(ph == (x.admitted ? 1 : 0), "cancel of %lld reports phase %d", id, ph);
                CHECK(sch.resident_bytes() == bytes - (x.admitted ? x.bytes : 0), "bytes after cancel");
                CHECK(sch.find(id) == nullptr && sch.cancel(id) == -1, "cancelled request still known");
                if (!x.admitted) {
                    auto pos = std::find(submitted.begin() + next_admit, submitted.end(), id);
                    CHECK(pos != submitted.end(), "cancelled waiting request not queued");
                    submitted.erase(pos);
                }
                x.finished = true;
                ++finished;
            }
        }
        const std::vector<long long> admitted = sch.admit();
        for (long long id : admitted) {
            CHECK(next_admit < submitted.size() && submitted[next_admit] == id, "admission out of order (id %lld)", id);
            ++next_admit;
            t[id].admitted = true;
        }
        // now and then the device has no room for the last admissions: they go
        // back to the head of the queue and the cap falls
        if (!admitted.empty() && rng() % 10 == 0) {
            const size_t from = rng() % admitted.size();
            const std::vector<long long> back(admitted.begin() + (long)from, admitted.end());
            const long long bytes = sch.resident_bytes();
            long long back_bytes = 0;
            for (long long id : back) back_bytes += t[id].bytes, t[id].admitted = false;
            sch.unadmit(back);
            next_admit -= back.size();
            CHECK(sch.resident_bytes() == bytes - back_bytes, "bytes after unadmit");
            CHECK(sch.lim().cap_bytes == std::max(sch.resident_bytes(), t[back.front()].bytes), "cap after unadmit");
            const std::vector<long long> w = sch.waiting_ids();
            CHECK(w.size() >= back.size() && std::equal(back.begin(), back.end(), w.begin()), "unadmitted order");
        }
        const long long cap_now = sch.lim().cap_bytes;
        CHECK(sch.resident_bytes() <= cap_now || sch.n_running() <= 1, "resident %lld over cap %lld with %zu running",
              sch.resident_bytes(), cap_now, sch.n_running());
        iteration_plan p = sch.plan();
        long long tiles = 0;
        for (long long id : p.active) {
            CHECK(t[id].admitted && !t[id].finished, "inactive request %lld planned", id);
            tiles += (t[id].steps - t[id].done) > 0 ? t[id].tiles : 0;
        }
        CHECK(tiles <= budget || p.active.size() == 1, "tiles %lld over budget %lld with %zu active", tiles, budget,
              p.active.size());
        std::map<long long, int> rounds_here;
        CHECK((int)p.rounds.size() <= RULES, "rounds for %zu rule ids", p.rounds.size());
        for (int r = 0; r < (int)p.rounds.size(); ++r)
            for (size_t q = 0; q < p.rounds[r].size(); ++q)
                for (const round_entry& e : p.rounds[r][q]) {
                    truth& x = t[e.id];
                    CHECK(x.rule == r, "request %lld in the wrong rule group", e.id);
                    CHECK((int)q == rounds_here[e.id], "request %lld rounds out of order", e.id);
                    rounds_here[e.id]++;
                    CHECK(e.steps >= 1 && e.steps <= x.k, "round of %d steps with k=%d", e.steps, x.k);
                    CHECK(e.src == x.cur, "request %lld reads buffer %d, state is in %d", e.id, e.src, x.cur);
                    CHECK(e.tpar == ((x.t0 + x.done) & 1), "request %lld step parity", e.id);
                    x.cur ^= 1;
                    x.done += e.steps;
                    x.rounds++;
                    CHECK(x.done <= x.steps, "request %lld overshoots", e.id);
                }
        for (long long id : p.active) CHECK(rounds_here[id] <= chunk_rounds, "more rounds than the chunk");
        for (const finish_entry& f : p.finishing) {
            truth& x = t[f.id];
            CHECK(!x.finished && x.done == x.steps, "request %lld finishes early or twice", f.id);
            CHECK(f.cur == (x.rounds & 1) && f.cur == x.cur, "request %lld final buffer", f.id);
            CHECK(f.keep == x.keep, "keep flag");
            x.finished = true;
            ++finished;
            if (x.keep) CHECK(sch.release(f.id), "release of kept request %lld", f.id);
            else CHECK(!sch.release(f.id), "unkept request %lld still known", f.id);
        }
    }
    CHECK(finished == 300, "only %d of 300 requests finished", finished);
    CHECK(sch.resident_bytes() == 0 && sch.n_running() == 0 && sch.n_waiting() == 0, "leftovers");
    return 0;
}

int main() {
    scenario(1, 1000, 60, 4);
    scenario(2, 100, 1, 1);       // one tile: one request per iteration
    scenario(3, 1LL << 40, 1 << 20, 8);  // nothing binds
    scenario(4, 10, 5, 2);        // tight cap: most requests larger than a third of it
    std::printf("ok\n");
    return 0;
}
