// Three automata that neither the reference nor this library ships, written in
// the rule DSL the way the reference's src/<automaton>/algorithm.hpp and
// config.hpp are.  The header includes only core/ast.hpp and
// memory/state_dictionary.hpp, so it compiles against either header tree:
//   * against this library's tree with nvcc, instantiated outside the library
//     (tests/cpp/custom_rules_gpu.cu, the header-only custom-rule path);
//   * against the reference's tree with g++, run by the reference's own
//     standard evaluator (oracle/ref_custom.cpp), which checks the GPU results.
// Together they exercise Moore counts against two targets (highlife), an
// elif chain over four states with range tests (star_wars), and von Neumann
// counts, modulo, a horizontal neighbour and alternate_algorithms (parity_shift).
#ifndef CELLATO_TEST_CUSTOM_RULES_HPP
#define CELLATO_TEST_CUSTOM_RULES_HPP

#include "core/ast.hpp"
#include "memory/state_dictionary.hpp"

// HighLife, B36/S23.
namespace highlife {
using namespace cellato::ast;

enum class cell { dead, alive };
using alive = state_constant<cell::alive>;
using dead = state_constant<cell::dead>;
using n_alive = count_neighbors<alive, moore_8_neighbors>;
using born = p<p<n_alive, equals, constant<3>>, or_, p<n_alive, equals, constant<6>>>;
using stays = p<p<n_alive, equals, constant<2>>, or_, p<n_alive, equals, constant<3>>>;

using algorithm = if_<p<current_state, equals, alive>>::then_<
                      if_<stays>::then_<alive>::else_<dead>
                  >::else_<
                      if_<born>::then_<alive>::else_<dead>
                  >;

struct config {
    static constexpr char name[] = "highlife";
    using cell_state = cell;
    using algorithm = highlife::algorithm;
    using state_dictionary = cellato::memory::grids::state_dictionary<cell::dead, cell::alive>;
};
}  // namespace highlife

// "Star Wars", the Generations rule 345/2/4: a live cell survives with 3-5 live
// neighbours, otherwise it decays through two dying states; a dead cell is
// born with exactly 2 live neighbours.
namespace star_wars {
using namespace cellato::ast;

enum class cell { dead, alive, dying_1, dying_2 };
using alive = state_constant<cell::alive>;
using dead = state_constant<cell::dead>;
using dying_1 = state_constant<cell::dying_1>;
using dying_2 = state_constant<cell::dying_2>;
using n_alive = count_neighbors<alive, moore_8_neighbors>;
using survives = p<p<n_alive, greater_than, constant<2>>, and_, p<n_alive, less_than, constant<6>>>;

using algorithm = if_<p<current_state, equals, alive>>::then_<
                      if_<survives>::then_<alive>::else_<dying_1>
                  >::elif_<p<current_state, equals, dying_1>>::then_<dying_2>
                  ::elif_<p<current_state, equals, dying_2>>::then_<dead>
                  ::else_<
                      if_<p<n_alive, equals, constant<2>>>::then_<alive>::else_<dead>
                  >;

struct config {
    static constexpr char name[] = "star-wars";
    using cell_state = cell;
    using algorithm = star_wars::algorithm;
    using state_dictionary = cellato::memory::grids::state_dictionary<cell::dead, cell::alive, cell::dying_1,
                                                                      cell::dying_2>;
};
}  // namespace star_wars

// On even steps Fredkin's parity rule on the von Neumann neighbourhood (a cell
// is on when an odd number of its four neighbours are on); on odd steps every
// cell takes the state of its left neighbour.
namespace parity_shift {
using namespace cellato::ast;

enum class cell { off, on };
using on = state_constant<cell::on>;
using off = state_constant<cell::off>;
using odd_neighbours =
    p<modulo<count_neighbors<on, von_neumann_4_neighbors>, constant<2>>, equals, constant<1>>;
using parity = if_<odd_neighbours>::then_<on>::else_<off>;
using shift = neighbor_at<-1, 0>;

using algorithm = alternate_algorithms<parity, shift>;

struct config {
    static constexpr char name[] = "parity-shift";
    using cell_state = cell;
    using algorithm = parity_shift::algorithm;
    using state_dictionary = cellato::memory::grids::state_dictionary<cell::off, cell::on>;
};
}  // namespace parity_shift

#endif  // CELLATO_TEST_CUSTOM_RULES_HPP
