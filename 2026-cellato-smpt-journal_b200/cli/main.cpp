// cellato -- command-line driver of the B200 bit-plane path.
//
// Same flags, suite selection, CSV line (stdout) and report (stderr) as the
// reference CLI (src/main.cpp:131-321, src/args-parser.hpp), restricted to the
// CUDA suites this library implements:
//   --device CUDA --traverser simple|temporal --evaluator bit_planes|tiled_bit_planes
//   --layout <same as evaluator> --word_size 32|64
//   --device CUDA --traverser simple --evaluator bit_array --layout bit_array
//   --word_size 32|64 (steps on bit planes; the grid converted on the device)
// e.g.  cellato --automaton wire --device CUDA --traverser temporal \
//         --evaluator tiled_bit_planes --layout tiled_bit_planes --word_size 64 \
//         --x_size 16384 --y_size 16384 --steps 1000 --temporal_steps 8 --temporal_tile_size_y 0
#include <algorithm>
#include <cstdint>
#include <iostream>
#include <string>
#include <vector>

#include "all.hpp"
#include "experiments/experiment_manager.hpp"
#include "experiments/run_params.hpp"
#include "experiments/test_suites.hpp"

namespace {

struct args {
    std::vector<std::string> tokens;
    args(int argc, char** argv) : tokens(argv + 1, argv + argc) {}
    bool exists(const std::string& o) const {
        return std::find(tokens.begin(), tokens.end(), "--" + o) != tokens.end();
    }
    std::string get(const std::string& o) const {
        auto it = std::find(tokens.begin(), tokens.end(), "--" + o);
        return (it != tokens.end() && it + 1 != tokens.end()) ? *(it + 1) : std::string();
    }
    int get_int(const std::string& o, int dflt) const { return exists(o) ? std::stoi(get(o)) : dflt; }
};

void usage() {
    std::cout << "Usage: cellato [options]\n"
                 "  --automaton <name>              game-of-life, forest-fire, wire, excitable, brian, maze,\n"
                 "                                  cyclic, fluid, critters, traffic\n"
                 "  --device CUDA                   (this library runs the CUDA bit-plane path)\n"
                 "  --traverser simple|temporal\n"
                 "  --evaluator bit_planes|tiled_bit_planes\n"
                 "  --layout bit_planes|tiled_bit_planes\n"
                 "  --word_size 32|64\n"
                 "  --x_size N --y_size N --steps N\n"
                 "  --temporal_steps K              steps fused per launch (temporal)\n"
                 "  --temporal_tile_size_y N        tile height in words, 0 = library choice (temporal)\n"
                 "  --rounds N --warmup_rounds N --seed N\n"
                 "  --print                         print the grid after each step\n"
                 "  --print_csv_header              print the CSV header and exit\n"
                 "  --cuda_block_size_x/_y N        accepted for compatibility, ignored\n";
}

template <typename... suites>
struct switch_ {
    static bool run(cellato::run::run_params& params) { return (call<suites>(params) || ...); }

    template <typename suite>
    static bool call(cellato::run::run_params& params) {
        if (!suite::is_for(params)) return false;
        using A = typename suite::automaton;
        auto initial = A::input::random::init(params);
        cellato::run::experiment_manager<suite> manager;
        auto report = manager.run_experiment(params, initial);
        std::cout << report.csv_line() << std::endl;
        report.pretty_print(std::cerr);
        return true;
    }
};

}  // namespace

int main(int argc, char** argv) {
    args a(argc, argv);
    if (a.exists("help")) {
        usage();
        return 0;
    }
    if (a.exists("print_csv_header")) {
        std::cout << cellato::run::experiment_report::csv_header() << std::endl;
        return 0;
    }
    std::vector<std::string> required{"automaton", "device", "traverser", "evaluator", "layout",
                                      "x_size",    "y_size", "steps",     "word_size"};
    if (a.get("traverser") == "temporal") required.push_back("temporal_steps");
    for (const auto& o : required)
        if (!a.exists(o)) {
            std::cerr << "Missing required option: " << o << std::endl;
            return 1;
        }
    cellato::run::run_params params;
    params.automaton = a.get("automaton");
    if (params.automaton == "fire") params.automaton = "forest-fire";
    params.device = a.get("device");
    params.traverser = a.get("traverser");
    params.evaluator = a.get("evaluator");
    params.layout = a.get("layout");
    params.x_size = a.get_int("x_size", 0);
    params.y_size = a.get_int("y_size", 0);
    params.steps = a.get_int("steps", 0);
    params.word_size = a.get_int("word_size", 0);
    params.temporal_steps = a.get_int("temporal_steps", 0);
    params.temporal_tile_size_y = a.get_int("temporal_tile_size_y", 0);
    params.rounds = a.get_int("rounds", 1);
    params.warmup_rounds = a.get_int("warmup_rounds", 0);
    params.seed = a.get_int("seed", 42);
    params.print = a.exists("print");
    params.cuda_block_size_x = a.get_int("cuda_block_size_x", 32);
    params.cuda_block_size_y = a.get_int("cuda_block_size_y", 8);

    namespace test = cellato::run::test_suites::on_cuda;
#define CELLATO_CASES(A)                                                                                    \
    test::using_<std::uint32_t>::bit_planes<A>, test::using_<std::uint64_t>::bit_planes<A>,                 \
        test::using_<std::uint32_t>::tiled_bit_planes<A>, test::using_<std::uint64_t>::tiled_bit_planes<A>, \
        test::using_<std::uint32_t>::temporal_linear_bit_planes<A>,                                         \
        test::using_<std::uint64_t>::temporal_linear_bit_planes<A>,                                         \
        test::using_<std::uint32_t>::temporal_tiled_bit_planes<A>,                                          \
        test::using_<std::uint64_t>::temporal_tiled_bit_planes<A>,                                          \
        test::using_<std::uint32_t>::bit_array<A>, test::using_<std::uint64_t>::bit_array<A>
    try {
        const bool ran =
            switch_<CELLATO_CASES(game_of_life::config), CELLATO_CASES(fire::config), CELLATO_CASES(wire::config),
                    CELLATO_CASES(excitable::config), CELLATO_CASES(brian::config), CELLATO_CASES(maze::config),
                    CELLATO_CASES(cyclic::config), CELLATO_CASES(fluid::config), CELLATO_CASES(critters::config),
                    CELLATO_CASES(traffic::config)>::run(params);
        if (!ran) {
            std::cerr << "No suitable test suite found for the given parameters." << std::endl;
            return 2;
        }
    } catch (const std::exception& e) {
        std::cerr << e.what() << std::endl;
        return 3;
    }
    return 0;
}
