// Scheduling policy of the simulation server (cellato_server_*): admission by
// device footprint, activation by a per-round tile budget, and the plan of one
// continuous-batching iteration.  Host-only C++ with no CUDA dependency, so the
// policy is unit-tested on its own.
//
// A request is a grid of one automaton to be advanced `steps` steps, numbered
// from its start step t0 (0 for a new simulation, the step reached for one
// resumed from a snapshot; the reference runs one such grid per traverser call,
// include/traversers/cuda/temporal.cu:227-262; there is no server).  Its life:
//   waiting   -- submitted, no device memory yet;
//   resident  -- admitted: both plane buffers allocated and initialised.
//                Admission is strict FIFO in submission order while the
//                resident bytes stay within the cap, so a large request is
//                never overtaken and cannot starve;
//   finished  -- every step planned; the result is in buffer `cur`.
// Each iteration activates resident requests in admission order, first fit,
// while the sum of their tiles stays within the budget (the oldest one always
// runs), and advances each active request by up to chunk_rounds rounds of k
// steps (k per automaton).  Round r of an iteration covers the tiles of every
// active request of an automaton that has an r-th round; the device runs all
// rounds of one automaton in one persistent launch.  Each request's rounds
// carry its own step parity and ping-pong buffer, so requests admitted at
// different times share launches.
#ifndef CELLATO_B200_SERVE_SCHEDULE_HPP
#define CELLATO_B200_SERVE_SCHEDULE_HPP

#include <algorithm>
#include <cstdint>
#include <deque>
#include <unordered_map>
#include <vector>

namespace cellato::b200::serve {

enum class phase : int { waiting = 0, resident = 1, finished = 2 };

struct request {
    long long id = 0;
    int rule = 0, x = 0, y = 0, steps = 0;
    int t0 = 0;           // number of its first step (only the parity matters to the rules)
    long long bytes = 0;  // device footprint of both plane buffers
    int tiles = 0;        // temporal tiles per round
    bool keep = false;    // planes stay after finishing until released
    int done = 0;         // steps planned so far
    int cur = 0;          // buffer (0 = a, 1 = b) holding the state after `done` steps
    phase ph = phase::waiting;
};

// One request's share of one round.
struct round_entry {
    long long id;
    int steps;  // 1..k
    int src;    // buffer read by this round
    int tpar;   // parity of the first step number of this round
};

// A request whose last step is planned in this iteration.
struct finish_entry {
    long long id;
    int cur;    // buffer holding its result
    bool keep;  // its planes stay until released
};

struct iteration_plan {
    std::vector<std::vector<std::vector<round_entry>>> rounds;  // rounds[rule][r] (rules seen so far)
    std::vector<long long> active;                        // requests advanced (admission order)
    std::vector<finish_entry> finishing;
    long long cell_steps = 0;
    int tiles = 0;
    bool empty() const { return active.empty(); }
};

struct limits {
    long long cap_bytes = 0;    // resident bytes allowed
    long long tile_budget = 1;  // tiles per round over all active requests
    int chunk_rounds = 4;       // rounds per request per iteration
    std::vector<int> k;         // steps per round by rule id; missing or 0 entries: 16
    int k_of(int rule) const {
        const int v = rule >= 0 && rule < (int)k.size() ? k[rule] : 0;
        return std::max(1, std::min(v > 0 ? v : 16, 32));
    }
};

class scheduler {
public:
    explicit scheduler(const limits& l) : lim_(l) {}

    const limits& lim() const { return lim_; }

    long long submit(int rule, int x, int y, int steps, long long bytes, int tiles, bool keep, int t0 = 0) {
        request r;
        r.id = next_id_++;
        r.rule = rule, r.x = x, r.y = y, r.steps = steps, r.t0 = t0;
        r.bytes = bytes, r.tiles = tiles, r.keep = keep;
        reqs_[r.id] = r;
        waiting_.push_back(r.id);
        return r.id;
    }

    // Admits waiting requests in submission order while they fit; returns them.
    // A request larger than the whole cap is admitted alone once nothing else
    // is resident (it can never fit otherwise).
    std::vector<long long> admit() {
        std::vector<long long> out;
        while (!waiting_.empty()) {
            request& r = reqs_[waiting_.front()];
            const bool fits = resident_bytes_ + r.bytes <= lim_.cap_bytes;
            if (!fits && !(resident_bytes_ == 0 && r.bytes > lim_.cap_bytes)) break;
            waiting_.pop_front();
            r.ph = phase::resident;
            resident_bytes_ += r.bytes;
            order_.push_back(r.id);
            out.push_back(r.id);
        }
        return out;
    }

    // Plans one iteration and advances the bookkeeping as if it had run.
    // Finishing requests without `keep` leave the resident total at once (the
    // caller frees their memory, stream-ordered, in the same iteration).
    iteration_plan plan() {
        iteration_plan p;
        long long used = 0;
        std::deque<long long> still;
        for (long long id : order_) {
            request& r = reqs_[id];
            const int left = r.steps - r.done;
            const int k = lim_.k_of(r.rule);
            const int chunk = std::min(left, lim_.chunk_rounds * k);
            const long long t = chunk > 0 ? r.tiles : 0;
            if (!p.active.empty() && used + t > lim_.tile_budget) {
                still.push_back(id);
                continue;
            }
            used += t;
            p.active.push_back(id);
            if ((int)p.rounds.size() <= r.rule) p.rounds.resize(r.rule + 1);
            auto& rr = p.rounds[r.rule];
            for (int s = 0, q = 0; s < chunk; s += k, ++q) {
                const int n = std::min(k, chunk - s);
                if ((int)rr.size() <= q) rr.emplace_back();
                rr[q].push_back(round_entry{id, n, r.cur, (r.t0 + r.done) & 1});
                r.cur ^= 1;
                r.done += n;
                p.cell_steps += (long long)r.x * r.y * n;
            }
            if (r.done == r.steps) {
                r.ph = phase::finished;
                p.finishing.push_back(finish_entry{id, r.cur, r.keep});
                if (!r.keep) drop(id);
            } else {
                still.push_back(id);
            }
        }
        p.tiles = (int)used;
        order_.swap(still);
        return p;
    }

    // Back-pressure from the device: requests just admitted (in admission
    // order) that could not get their memory go back to the head of the
    // waiting queue in the same order, and the cap falls to the bytes still
    // resident (at least the head request's), so admission waits for resident
    // requests to finish.
    void unadmit(const std::vector<long long>& ids) {
        if (ids.empty()) return;
        for (auto it = ids.rbegin(); it != ids.rend(); ++it) {
            request& r = reqs_[*it];
            r.ph = phase::waiting;
            resident_bytes_ -= r.bytes;
            order_.erase(std::find(order_.begin(), order_.end(), *it));
            waiting_.push_front(*it);
        }
        lim_.cap_bytes = std::max(resident_bytes_, reqs_[ids.front()].bytes);
    }

    // Forgets a finished request; returns false when it is unknown or not finished.
    bool release(long long id) {
        auto it = reqs_.find(id);
        if (it == reqs_.end() || it->second.ph != phase::finished) return false;
        if (it->second.keep) resident_bytes_ -= it->second.bytes;
        reqs_.erase(it);
        return true;
    }

    // Removes a request at any stage (preemption); its bytes leave the resident
    // total.  Returns the phase it was in, or -1 when it is unknown.
    int cancel(long long id) {
        auto it = reqs_.find(id);
        if (it == reqs_.end()) return -1;
        const request& r = it->second;
        const int ph = (int)r.ph;
        if (r.ph == phase::waiting) {
            waiting_.erase(std::find(waiting_.begin(), waiting_.end(), id));
        } else if (r.ph == phase::resident) {
            order_.erase(std::find(order_.begin(), order_.end(), id));
            resident_bytes_ -= r.bytes;
        } else if (r.keep) {
            resident_bytes_ -= r.bytes;
        }
        reqs_.erase(it);
        return ph;
    }

    const request* find(long long id) const {
        auto it = reqs_.find(id);
        return it == reqs_.end() ? nullptr : &it->second;
    }

    long long resident_bytes() const { return resident_bytes_; }
    size_t n_waiting() const { return waiting_.size(); }
    size_t n_running() const { return order_.size(); }  // resident, not finished
    std::vector<long long> waiting_ids() const { return {waiting_.begin(), waiting_.end()}; }
    std::vector<long long> running_ids() const { return {order_.begin(), order_.end()}; }

private:
    // a finished request that keeps no planes: its bytes leave, its record goes
    void drop(long long id) {
        resident_bytes_ -= reqs_[id].bytes;
        reqs_.erase(id);
    }

    limits lim_;
    long long next_id_ = 1;
    long long resident_bytes_ = 0;
    std::unordered_map<long long, request> reqs_;
    std::deque<long long> waiting_;  // submission order
    std::deque<long long> order_;    // resident and running, admission order
};

}  // namespace cellato::b200::serve

#endif  // CELLATO_B200_SERVE_SCHEDULE_HPP
