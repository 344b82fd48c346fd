// Test harness (host build): the reference's own automaton headers
// (src/<automaton>/config.hpp, found through the reference source tree on the
// include path) compiled against this library's header tree (core/ast.hpp,
// memory/, experiments/, traversers/cuda_utils.cuh) and lowered by
// b200/lower.cuh.  If the rule DSL is source compatible this compiles, and the
// lowered rules reproduce the reference's results.
#include <cstdint>
#include <vector>

#include "b200/lower.cuh"
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

using namespace cellato::b200;

namespace {
template <class A>
int run(const uint8_t* in, uint8_t* out, int X, int Y, int steps) {
    using dict = typename A::state_dictionary;
    using net = rule_net<dict, typename A::algorithm>;
    constexpr int NB = dict::needed_bits;
    if (X % 32) return -1;
    const int Xw = X / 32;
    std::vector<word> cur(std::size_t(NB) * Xw * Y, 0), nxt(cur.size());
    auto P = [&](std::vector<word>& g, int p, int x, int y) -> word& { return g[(std::size_t(p) * Y + y) * Xw + x]; };
    for (int y = 0; y < Y; ++y)
        for (int x = 0; x < X; ++x)
            for (int p = 0; p < NB; ++p)
                if ((in[std::size_t(y) * X + x] >> p) & 1) P(cur, p, x / 32, y) |= word(1) << (x % 32);
    for (int t = 0; t < steps; ++t) {
        for (int y = 0; y < Y; ++y)
            for (int x = 0; x < Xw; ++x) {
                typename net::feat f[3];
                for (int dy = -1; dy <= 1; ++dy) {
                    const int yy = (y + dy + Y) % Y;
                    word C[NB], L[NB], R[NB];
                    for (int p = 0; p < NB; ++p) {
                        C[p] = P(cur, p, x, yy);
                        L[p] = P(cur, p, (x + Xw - 1) % Xw, yy);
                        R[p] = P(cur, p, (x + 1) % Xw, yy);
                    }
                    f[dy + 1] = net::make_feat(C, L, R);
                }
                word o[NB];
                if (t & 1)
                    net::template eval<1>(f[0], f[1], f[2], y & 1, o);
                else
                    net::template eval<0>(f[0], f[1], f[2], y & 1, o);
                for (int p = 0; p < NB; ++p) P(nxt, p, x, y) = o[p];
            }
        std::swap(cur, nxt);
    }
    for (int y = 0; y < Y; ++y)
        for (int x = 0; x < X; ++x) {
            uint8_t v = 0;
            for (int p = 0; p < NB; ++p) v |= uint8_t(((P(cur, p, x / 32, y) >> (x % 32)) & 1) << p);
            out[std::size_t(y) * X + x] = v;
        }
    return 0;
}
}  // namespace

extern "C" int reference_rules_lowered_run(int rule, const uint8_t* in, uint8_t* out, int X, int Y, int steps) {
    switch (rule) {
        case 0: return run<game_of_life::config>(in, out, X, Y, steps);
        case 1: return run<fire::config>(in, out, X, Y, steps);
        case 2: return run<wire::config>(in, out, X, Y, steps);
        case 3: return run<excitable::config>(in, out, X, Y, steps);
        case 4: return run<brian::config>(in, out, X, Y, steps);
        case 5: return run<maze::config>(in, out, X, Y, steps);
        case 6: return run<cyclic::config>(in, out, X, Y, steps);
        case 7: return run<fluid::config>(in, out, X, Y, steps);
        case 8: return run<critters::config>(in, out, X, Y, steps);
        case 9: return run<traffic::config>(in, out, X, Y, steps);
    }
    return -1;
}
