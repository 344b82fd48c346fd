// Test infrastructure only: the reference's own, unmodified CPU standard path
// (evaluators::standard + traversers::cpu::simple, include/evaluators/
// standard.hpp:25-285, include/traversers/cpu/simple.hpp:42-88) instantiated
// for the custom rules of tests/cpp/custom_rules.hpp, which are not part of
// the reference.  Compiled by oracle/Makefile against the reference's header
// tree into oracle/_ref/.  The tests compare the B200 library's runs of the
// same rule source (instantiated outside the library) with these results, and
// tests/golden/make_golden.py records them as fixtures.
#include <cstdint>
#include <vector>

#include "experiments/run_params.hpp"
#include "evaluators/standard.hpp"
#include "memory/standard_grid.hpp"
#include "traversers/cpu/simple.hpp"

#include "custom_rules.hpp"

namespace {

template <typename A>
int run_standard(const uint8_t* in, uint8_t* out, int X, int Y, int steps) {
    using cell_t = typename A::cell_state;
    using dict = typename A::state_dictionary;
    using grid_t = cellato::memory::grids::standard::grid<cell_t>;
    using eval_t = cellato::evaluators::standard::evaluator<cell_t, typename A::algorithm>;
    using trav_t = cellato::traversers::cpu::simple::traverser<eval_t, grid_t>;
    const std::size_t n = std::size_t(X) * Y;
    std::vector<cell_t> st(n);
    for (std::size_t i = 0; i < n; ++i) st[i] = dict::index_to_state(in[i]);
    grid_t g(std::move(st), X, Y);
    cellato::run::run_params params;
    params.x_size = X;
    params.y_size = Y;
    params.steps = steps;
    trav_t trav;
    trav.init(g, params);
    trav.run(steps);
    grid_t res = trav.fetch_result();
    for (std::size_t i = 0; i < n; ++i) out[i] = static_cast<uint8_t>(dict::state_to_index(res.data()[i]));
    return 0;
}

}  // namespace

extern "C" {

int cref_custom_count() { return 3; }

const char* cref_custom_name(int which) {
    switch (which) {
        case 0: return highlife::config::name;
        case 1: return star_wars::config::name;
        case 2: return parity_shift::config::name;
        default: return nullptr;
    }
}

int cref_custom_states(int which) {
    switch (which) {
        case 0: return highlife::config::state_dictionary::number_of_values;
        case 1: return star_wars::config::state_dictionary::number_of_values;
        case 2: return parity_shift::config::state_dictionary::number_of_values;
        default: return -1;
    }
}

// `steps` steps of custom rule `which` from step 0; cells are dictionary indices.
int cref_custom_run(int which, const uint8_t* in, uint8_t* out, int X, int Y, int steps) {
    switch (which) {
        case 0: return run_standard<highlife::config>(in, out, X, Y, steps);
        case 1: return run_standard<star_wars::config>(in, out, X, Y, steps);
        case 2: return run_standard<parity_shift::config>(in, out, X, Y, steps);
        default: return -1;
    }
}

}  // extern "C"
