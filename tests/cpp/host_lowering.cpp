// Test harness (host build): runs the B200 rule lowering (b200/lower.cuh) on
// the CPU over linear 32-bit plane words with torus wrap, so the lowering of
// every rule can be checked against the oracle without a GPU.  This is test
// infrastructure; the product only runs the lowering inside its CUDA kernels.
#include <cstdint>
#include <cstring>
#include <vector>

#include "b200/lower.cuh"
#include "all.hpp"

using namespace cellato::b200;

namespace {

template <class A>
int run(const uint8_t* in, uint8_t* out, int X, int Y, int t0, int steps) {
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
    for (int s = 0; s < steps; ++s) {
        const int t = t0 + s;
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

extern "C" int host_lowered_run(int rule, const uint8_t* in, uint8_t* out, int X, int Y, int t0, int steps) {
    switch (rule) {
        case 0: return run<game_of_life::config>(in, out, X, Y, t0, steps);
        case 1: return run<fire::config>(in, out, X, Y, t0, steps);
        case 2: return run<wire::config>(in, out, X, Y, t0, steps);
        case 3: return run<excitable::config>(in, out, X, Y, t0, steps);
        case 4: return run<brian::config>(in, out, X, Y, t0, steps);
        case 5: return run<maze::config>(in, out, X, Y, t0, steps);
        case 6: return run<cyclic::config>(in, out, X, Y, t0, steps);
        case 7: return run<fluid::config>(in, out, X, Y, t0, steps);
        case 8: return run<critters::config>(in, out, X, Y, t0, steps);
        case 9: return run<traffic::config>(in, out, X, Y, t0, steps);
    }
    return -1;
}

// The seeded initial grid of each automaton config (config::input::random,
// what the cellato CLI starts from), as dictionary indices.
template <class A>
int config_init(int X, int Y, int seed, uint8_t* out) {
    cellato::run::run_params params;
    params.x_size = X;
    params.y_size = Y;
    params.seed = seed;
    const auto st = A::input::random::init(params);
    for (std::size_t i = 0; i < st.size(); ++i) out[i] = (uint8_t)A::state_dictionary::state_to_index(st[i]);
    return 0;
}

extern "C" int host_config_init(int rule, int X, int Y, int seed, uint8_t* out) {
    switch (rule) {
        case 0: return config_init<game_of_life::config>(X, Y, seed, out);
        case 1: return config_init<fire::config>(X, Y, seed, out);
        case 2: return config_init<wire::config>(X, Y, seed, out);
        case 3: return config_init<excitable::config>(X, Y, seed, out);
        case 4: return config_init<brian::config>(X, Y, seed, out);
        case 5: return config_init<maze::config>(X, Y, seed, out);
        case 6: return config_init<cyclic::config>(X, Y, seed, out);
        case 7: return config_init<fluid::config>(X, Y, seed, out);
        case 8: return config_init<critters::config>(X, Y, seed, out);
        case 9: return config_init<traffic::config>(X, Y, seed, out);
    }
    return -1;
}
