// Run parameters of the cellato CLI; same fields, defaults and CSV columns as
// the reference include/experiments/run_params.hpp:10-97, so scripts that parse
// the CLI's CSV lines keep working.
#ifndef RUN_PARAMS_HPP
#define RUN_PARAMS_HPP

#include <cstddef>
#include <iostream>
#include <string>

namespace cellato::run {

struct run_params {
    std::string automaton = "game-of-life";
    std::string device = "CPU";
    std::string traverser = "standard";
    std::string evaluator = "standard";
    std::string layout = "standard";
    std::string reference_impl = "none";

    int x_size = 0;
    int y_size = 0;
    int steps = 0;
    int word_size = 0;
    int x_tile_size = 0;
    int y_tile_size = 0;
    int temporal_steps = 0;
    int temporal_tile_size_y = 0;
    int rounds = 1;
    int warmup_rounds = 0;
    int seed = 42;

    bool print = false;
    bool help = false;
    bool print_csv_header = false;

    int cuda_block_size_x = 32;
    int cuda_block_size_y = 8;

    void print_to(std::ostream& os) const {
        os << "Run Parameters:\n"
           << "  Automaton: " << automaton << "\n  Device: " << device << "\n  Traverser: " << traverser
           << "\n  Evaluator: " << evaluator << "\n  Layout: " << layout << "\n  Reference Implementation: "
           << reference_impl << "\n  Grid Size: (" << x_size << ", " << y_size << ")\n  Steps: " << steps
           << "\n  Word Size: " << word_size << "\n  Rounds: " << rounds << "\n  Warmup Rounds: " << warmup_rounds
           << "\n  Seed: " << seed << "\n  Temporal Steps: " << temporal_steps
           << "\n  Temporal Tile Size Y: " << temporal_tile_size_y << "\n  CUDA Block Size: (" << cuda_block_size_x
           << ", " << cuda_block_size_y << ")\n";
    }
    void print_std() const { print_to(std::cout); }

    static std::string csv_header() {
        return "automaton,device,traverser,evaluator,layout,reference_impl,x_size,y_size,steps,rounds,warmup_rounds,"
               "x_tile_size,y_tile_size,cuda_block_size_x,cuda_block_size_y,seed,word_size,temporal_steps,"
               "temporal_tile_size_y";
    }

    std::string csv_line() const {
        auto s = [](int v) { return std::to_string(v); };
        return automaton + "," + device + "," + traverser + "," + evaluator + "," + layout + "," +
               (reference_impl != "none" ? reference_impl : std::string()) + "," + s(x_size) + "," + s(y_size) +
               "," + s(steps) + "," + s(rounds) + "," + s(warmup_rounds) + "," + s(x_tile_size) + "," +
               s(y_tile_size) + "," + s(cuda_block_size_x) + "," + s(cuda_block_size_y) + "," + s(seed) + "," +
               s(word_size) + "," + s(temporal_steps) + "," + s(temporal_tile_size_y);
    }
};

}  // namespace cellato::run

#endif  // RUN_PARAMS_HPP
