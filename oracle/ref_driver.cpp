// Test infrastructure only: a thin extern "C" driver around the reference's
// own, unmodified CPU code for the bit-plane hot path.  It is compiled from the
// reference headers where they lie (include/ and src/ of the reference tree,
// read-only include paths) by oracle/Makefile into oracle/_ref/.  Only the
// tests, __graft_entry__.smoke() and bench.py's CPU-baseline leg load it, and
// only as the checker or as the timed CPU baseline -- never as the product.
//
// What it wraps (reference file:line):
//   * CPU standard path: evaluators::standard + traversers::cpu::simple
//     (include/evaluators/standard.hpp:25-285,
//      include/traversers/cpu/simple.hpp:42-88, selected by
//      include/experiments/test_suites.hpp:233-257).
//   * CPU bit_planes / tiled_bit_planes paths (same traverser, the
//     bit-plane evaluators include/evaluators/bit_planes.hpp:45-663 and
//     include/evaluators/tiled_bit_planes.hpp:60-396) -- a secondary check.
//   * grid packing of include/memory/bit_planes_grid.hpp:234-270,
//     include/memory/tiled_bit_planes_grid.hpp:243-288 and
//     include/memory/bit_array_grid.hpp:143-159, 298-310, used to pin layouts.
//   * the reference's seeded initialisers src/<automaton>/data_init.hpp.
//   * the 4x4 tile-sum checksum include/memory/standard_grid.hpp:179-213.
//
// Cell values cross this ABI as uint8 *dictionary indices* (the value a bit
// plane encodes), never as raw enum values; the driver maps them through each
// automaton's state_dictionary (include/memory/state_dictionary.hpp:10-70).

#include <algorithm>
#include <barrier>
#include <cstdint>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "experiments/run_params.hpp"
#include "evaluators/standard.hpp"
#include "evaluators/bit_planes.hpp"
#include "evaluators/tiled_bit_planes.hpp"
#include "memory/standard_grid.hpp"
#include "memory/bit_planes_grid.hpp"
#include "memory/tiled_bit_planes_grid.hpp"
#include "memory/bit_array_grid.hpp"
#include "traversers/cpu/simple.hpp"
#include "traversers/traverser_utils.hpp"

#include "game_of_life/config.hpp"
#include "fire/config.hpp"
#include "wire/config.hpp"
#include "excitable/config.hpp"
#include "brian/config.hpp"
#include "maze/config.hpp"
#include "cyclic/config.hpp"
#include "fluid/config.hpp"
#include "critters/config.hpp"
#include "traffic/config.hpp"

namespace {

namespace grids = cellato::memory::grids;
namespace evals = cellato::evaluators;

template <typename A>
using cell_of = typename A::cell_state;

template <typename A>
std::vector<cell_of<A>> to_states(const uint8_t* idx, std::size_t n) {
    std::vector<cell_of<A>> out(n);
    for (std::size_t i = 0; i < n; ++i)
        out[i] = A::state_dictionary::index_to_state(idx[i]);
    return out;
}

template <typename A>
void to_indices(const cell_of<A>* st, std::size_t n, uint8_t* out) {
    for (std::size_t i = 0; i < n; ++i)
        out[i] = static_cast<uint8_t>(A::state_dictionary::state_to_index(st[i]));
}

// The reference CPU standard path exactly as the cellato CLI runs it
// (experiment_manager -> cpu::simple::traverser::init/run/fetch_result).
template <typename A>
int run_standard(const uint8_t* in, uint8_t* out, int X, int Y, int steps) {
    using cell_t = cell_of<A>;
    using grid_t = grids::standard::grid<cell_t>;
    using eval_t = evals::standard::evaluator<cell_t, typename A::algorithm>;
    using trav_t = cellato::traversers::cpu::simple::traverser<eval_t, grid_t>;
    const std::size_t n = std::size_t(X) * Y;
    auto st = to_states<A>(in, n);
    grid_t g(std::move(st), X, Y);
    cellato::run::run_params params;
    params.x_size = X;
    params.y_size = Y;
    params.steps = steps;
    trav_t trav;
    trav.init(g, params);
    trav.run(steps);
    grid_t res = trav.fetch_result();
    to_indices<A>(res.data(), n, out);
    return 0;
}

// Row-partitioned multi-threaded driver that calls the reference standard
// evaluator unchanged, one cell per call, exactly as
// include/traversers/cpu/simple.hpp:60-85 does; rows are split over threads
// and a barrier separates steps.  Used for the all-cores CPU baseline.
template <typename A>
int run_standard_mt(const uint8_t* in, uint8_t* out, int X, int Y, int steps, int threads) {
    using cell_t = cell_of<A>;
    using eval_t = evals::standard::evaluator<cell_t, typename A::algorithm>;
    const std::size_t n = std::size_t(X) * Y;
    std::vector<cell_t> a = to_states<A>(in, n), b(a);
    if (threads < 1) threads = 1;
    if (threads > Y) threads = Y;
    std::barrier sync(threads);
    auto worker = [&](int tid) {
        cell_t* cur = a.data();
        cell_t* nxt = b.data();
        const int y0 = int((long long)Y * tid / threads);
        const int y1 = int((long long)Y * (tid + 1) / threads);
        for (int step = 0; step < steps; ++step) {
            grids::point_in_grid<cell_t*> state{};
            state.grid = cur;
            state.properties.x_size = X;
            state.properties.y_size = Y;
            state.time_step = step;
            for (int y = y0; y < y1; ++y) {
                for (int x = 0; x < X; ++x) {
                    state.position.x = x;
                    state.position.y = y;
                    auto r = eval_t::evaluate(state);
                    cellato::traversers::utils::save_to(nxt, state.idx(), r);
                }
            }
            std::swap(cur, nxt);
            sync.arrive_and_wait();
        }
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < threads; ++t) pool.emplace_back(worker, t);
    worker(0);
    for (auto& t : pool) t.join();
    const cell_t* res = (steps % 2 == 0) ? a.data() : b.data();
    to_indices<A>(res, n, out);
    return 0;
}

// Reference CPU bit_planes / tiled_bit_planes evaluators under the CPU
// traverser (test_suites.hpp:342-383 family, on_cpu::using_<W>).
template <typename A, typename W, bool tiled>
int run_bit_planes(const uint8_t* in, uint8_t* out, int X, int Y, int steps) {
    using cell_t = cell_of<A>;
    using dict_t = typename A::state_dictionary;
    using grid_t = std::conditional_t<tiled, grids::tiled_bit_planes::grid<W, dict_t>,
                                      grids::bit_planes::grid<W, dict_t>>;
    using eval_t = std::conditional_t<tiled,
                                      evals::tiled_bit_planes::evaluator<W, dict_t, typename A::algorithm>,
                                      evals::bit_planes::evaluator<W, dict_t, typename A::algorithm>>;
    using trav_t = cellato::traversers::cpu::simple::traverser<eval_t, grid_t>;
    const std::size_t n = std::size_t(X) * Y;
    auto st = to_states<A>(in, n);
    grids::standard::grid<cell_t> sg(std::move(st), X, Y);
    grid_t g(sg);
    cellato::run::run_params params;
    params.x_size = X;
    params.y_size = Y;
    params.steps = steps;
    trav_t trav;
    trav.init(g, params);
    trav.run(steps);
    grid_t res = trav.fetch_result();
    auto sres = res.to_standard();
    to_indices<A>(sres.data(), n, out);
    return 0;
}

// Pack through the reference grid classes; planes_out receives nb arrays of
// (bytes_per_plane) bytes each, laid out back to back.
template <typename A, typename W, bool tiled>
long long pack(const uint8_t* in, int X, int Y, uint8_t* planes_out) {
    using cell_t = cell_of<A>;
    using dict_t = typename A::state_dictionary;
    using grid_t = std::conditional_t<tiled, grids::tiled_bit_planes::grid<W, dict_t>,
                                      grids::bit_planes::grid<W, dict_t>>;
    const std::size_t n = std::size_t(X) * Y;
    auto st = to_states<A>(in, n);
    grids::standard::grid<cell_t> sg(std::move(st), X, Y);
    grid_t g(sg);
    const std::size_t words = g.x_size_physical() * g.y_size_physical();
    auto ptrs = g.data();
    for (int p = 0; p < dict_t::needed_bits; ++p)
        std::memcpy(planes_out + p * words * sizeof(W), ptrs[p], words * sizeof(W));
    return (long long)(words * sizeof(W));
}

// Pack through the reference bit_array grid; words_out receives its words.
template <typename A, typename W>
long long pack_bit_array(const uint8_t* in, int X, int Y, uint8_t* words_out) {
    using cell_t = cell_of<A>;
    using grid_t = grids::bit_array::grid<typename A::state_dictionary, W>;
    const std::size_t n = std::size_t(X) * Y;
    auto st = to_states<A>(in, n);
    grids::standard::grid<cell_t> sg(std::move(st), X, Y);
    grid_t g(sg);
    const std::size_t words = (n + grid_t::cells_per_word - 1) / grid_t::cells_per_word;
    std::memcpy(words_out, g.raw_data(), words * sizeof(W));
    return (long long)(words * sizeof(W));
}

template <typename A>
int reference_init(int X, int Y, int seed, uint8_t* out) {
    cellato::run::run_params params;
    params.x_size = X;
    params.y_size = Y;
    params.seed = seed;
    auto st = A::input::random::init(params);
    to_indices<A>(st.data(), st.size(), out);
    return 0;
}

template <typename A>
int checksum(const uint8_t* in, int X, int Y, char* buf, int buflen) {
    auto st = to_states<A>(in, std::size_t(X) * Y);
    grids::standard::grid<cell_of<A>> g(std::move(st), X, Y);
    std::string s = g.get_checksum();
    if ((int)s.size() + 1 > buflen) return -1;
    std::memcpy(buf, s.c_str(), s.size() + 1);
    return (int)s.size();
}

template <typename A>
int state_value(int index) {
    return static_cast<int>(A::state_dictionary::index_to_state(index));
}

// Dispatch on the rule id used throughout this project:
// 0 game-of-life, 1 forest-fire, 2 wire, 3 excitable, 4 brian, 5 maze,
// 6 cyclic, 7 fluid, 8 critters, 9 traffic.
template <typename F>
int with_rule(int rule, F&& f) {
    switch (rule) {
        case 0: return f.template operator()<game_of_life::config>();
        case 1: return f.template operator()<fire::config>();
        case 2: return f.template operator()<wire::config>();
        case 3: return f.template operator()<excitable::config>();
        case 4: return f.template operator()<brian::config>();
        case 5: return f.template operator()<maze::config>();
        case 6: return f.template operator()<cyclic::config>();
        case 7: return f.template operator()<fluid::config>();
        case 8: return f.template operator()<critters::config>();
        case 9: return f.template operator()<traffic::config>();
        default: return -1;
    }
}

}  // namespace

extern "C" {

int cref_rule_count() { return 10; }

const char* cref_rule_name(int rule) {
    static const char* names[] = {game_of_life::config::name, fire::config::name, wire::config::name,
                                  excitable::config::name,    brian::config::name, maze::config::name,
                                  cyclic::config::name,       fluid::config::name, critters::config::name,
                                  traffic::config::name};
    return (rule >= 0 && rule < 10) ? names[rule] : nullptr;
}

int cref_needed_bits(int rule) {
    return with_rule(rule, []<typename A>() { return (int)A::state_dictionary::needed_bits; });
}

int cref_number_of_states(int rule) {
    return with_rule(rule, []<typename A>() { return (int)A::state_dictionary::number_of_values; });
}

int cref_state_value(int rule, int index) {
    return with_rule(rule, [index]<typename A>() { return state_value<A>(index); });
}

int cref_run_standard(int rule, const uint8_t* in, uint8_t* out, int X, int Y, int steps) {
    try {
        return with_rule(rule, [=]<typename A>() { return run_standard<A>(in, out, X, Y, steps); });
    } catch (...) {
        return -2;
    }
}

int cref_run_standard_mt(int rule, const uint8_t* in, uint8_t* out, int X, int Y, int steps, int threads) {
    try {
        return with_rule(rule, [=]<typename A>() { return run_standard_mt<A>(in, out, X, Y, steps, threads); });
    } catch (...) {
        return -2;
    }
}

int cref_run_bit_planes(int rule, int word_bits, int tiled, const uint8_t* in, uint8_t* out, int X, int Y,
                        int steps) {
    try {
        return with_rule(rule, [=]<typename A>() {
            if (word_bits == 32 && !tiled) return run_bit_planes<A, uint32_t, false>(in, out, X, Y, steps);
            if (word_bits == 64 && !tiled) return run_bit_planes<A, uint64_t, false>(in, out, X, Y, steps);
            if (word_bits == 32 && tiled) return run_bit_planes<A, uint32_t, true>(in, out, X, Y, steps);
            if (word_bits == 64 && tiled) return run_bit_planes<A, uint64_t, true>(in, out, X, Y, steps);
            return -1;
        });
    } catch (...) {
        return -2;
    }
}

long long cref_pack(int rule, int word_bits, int tiled, const uint8_t* in, int X, int Y, uint8_t* planes_out) {
    try {
        long long r = -1;
        with_rule(rule, [&]<typename A>() {
            if (word_bits == 32 && !tiled) r = pack<A, uint32_t, false>(in, X, Y, planes_out);
            if (word_bits == 64 && !tiled) r = pack<A, uint64_t, false>(in, X, Y, planes_out);
            if (word_bits == 32 && tiled) r = pack<A, uint32_t, true>(in, X, Y, planes_out);
            if (word_bits == 64 && tiled) r = pack<A, uint64_t, true>(in, X, Y, planes_out);
            return 0;
        });
        return r;
    } catch (...) {
        return -2;
    }
}

long long cref_pack_bit_array(int rule, int word_bits, const uint8_t* in, int X, int Y, uint8_t* words_out) {
    try {
        long long r = -1;
        with_rule(rule, [&]<typename A>() {
            if (word_bits == 32) r = pack_bit_array<A, uint32_t>(in, X, Y, words_out);
            if (word_bits == 64) r = pack_bit_array<A, uint64_t>(in, X, Y, words_out);
            return 0;
        });
        return r;
    } catch (...) {
        return -2;
    }
}

int cref_reference_init(int rule, int X, int Y, int seed, uint8_t* out) {
    try {
        return with_rule(rule, [=]<typename A>() { return reference_init<A>(X, Y, seed, out); });
    } catch (...) {
        return -2;
    }
}

int cref_checksum(int rule, const uint8_t* in, int X, int Y, char* buf, int buflen) {
    try {
        return with_rule(rule, [=]<typename A>() { return checksum<A>(in, X, Y, buf, buflen); });
    } catch (...) {
        return -2;
    }
}

}  // extern "C"
