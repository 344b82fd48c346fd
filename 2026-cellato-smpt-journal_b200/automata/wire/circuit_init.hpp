// The seeded WireWorld circuit the reference's CLI starts from
// (src/wire/data_init.hpp:11-216 of the reference), restated.  On an empty
// grid it lays conductor as
//   1. concentric rectangular loops around the centre, half-width s and
//      half-height s/2 for s = 4, 8, 12, ... while the loop fits;
//   2. ten straight runs of 10-30 cells (horizontal, vertical or diagonal);
//   3. five circles of radius 5-15, sampled every 5 degrees;
//   4. eight crossings: a 9-cell horizontal bar and a 9-cell vertical bar with
//      the centre cell left out, away from the border;
// then shuffles the list of every conductor cell laid (repeats included) and
// puts an electron -- a head, with a tail on a conductor among its four
// neighbours taken in shuffled order -- on every 20th entry of the list; a
// head without such a neighbour reverts to conductor.  Every random choice
// comes from one std::mt19937 seeded with the run's seed, drawn in the order
// above with the same standard distributions, so the same seed gives the same
// grid as the reference.  Runs and circles clip at the border; the grid does
// not wrap here.
#ifndef WIRE_CIRCUIT_INIT_HPP
#define WIRE_CIRCUIT_INIT_HPP

#include <algorithm>
#include <cmath>
#include <random>
#include <utility>
#include <vector>

#include "experiments/run_params.hpp"

namespace wire {

template <typename State>
class circuit_builder {
public:
    circuit_builder(int X, int Y, unsigned seed) : X_(X), Y_(Y), cells_(std::size_t(X) * Y, State::empty) {
        rng_.seed(seed);
    }

    std::vector<State> build() {
        loops();
        std::uniform_int_distribution<int> xs(0, X_ - 1), ys(0, Y_ - 1);
        runs(xs, ys);
        circles(xs, ys);
        crossings(xs, ys);
        electrons();
        return std::move(cells_);
    }

private:
    bool inside(int x, int y) const { return x >= 0 && x < X_ && y >= 0 && y < Y_; }
    State& at(int x, int y) { return cells_[std::size_t(y) * X_ + x]; }

    void lay(int x, int y) {
        at(x, y) = State::conductor;
        laid_.emplace_back(x, y);
    }

    // 1. nested 2:1 rectangles, every 4 cells, while they fit
    void loops() {
        const int cx = X_ / 2, cy = Y_ / 2;
        for (int w = 4; w <= std::max(cx, cy); w += 4) {
            const int h = w / 2;
            if (cx + w >= X_ || cx - w < 0 || cy + h >= Y_ || cy - h < 0) return;
            for (int x = cx - w; x <= cx + w; ++x) lay(x, cy - h);
            for (int x = cx - w; x <= cx + w; ++x) lay(x, cy + h);
            for (int y = cy - h + 1; y < cy + h; ++y) lay(cx - w, y);
            for (int y = cy - h + 1; y < cy + h; ++y) lay(cx + w, y);
        }
    }

    // 2. straight runs from random points in one of eight directions
    void runs(std::uniform_int_distribution<int>& xs, std::uniform_int_distribution<int>& ys) {
        std::uniform_int_distribution<int> lengths(10, 30);
        for (int n = 0; n < 10; ++n) {
            const int x0 = xs(rng_), y0 = ys(rng_);
            int dx = int(rng_() % 3) - 1;
            const int dy = int(rng_() % 3) - 1;
            if (dx == 0 && dy == 0) dx = 1;
            const int len = lengths(rng_);
            for (int j = 0; j < len; ++j)
                if (inside(x0 + j * dx, y0 + j * dy)) lay(x0 + j * dx, y0 + j * dy);
        }
    }

    // 3. circles sampled at 72 angles (truncated towards zero)
    void circles(std::uniform_int_distribution<int>& xs, std::uniform_int_distribution<int>& ys) {
        std::uniform_int_distribution<int> radii(5, 15);
        for (int n = 0; n < 5; ++n) {
            const int cx = xs(rng_), cy = ys(rng_), r = radii(rng_);
            for (int deg = 0; deg < 360; deg += 5) {
                const double a = deg * M_PI / 180.0;
                const int x = cx + static_cast<int>(r * std::cos(a));
                const int y = cy + static_cast<int>(r * std::sin(a));
                if (inside(x, y)) lay(x, y);
            }
        }
    }

    // 4. a horizontal bar crossed by a vertical bar with a gap at the centre
    void crossings(std::uniform_int_distribution<int>& xs, std::uniform_int_distribution<int>& ys) {
        for (int n = 0; n < 8; ++n) {
            const int x = xs(rng_), y = ys(rng_);
            if (!(x > 5 && x < X_ - 5 && y > 5 && y < Y_ - 5)) continue;
            for (int d = -4; d <= 4; ++d) lay(x + d, y);
            for (int d = -4; d <= 4; ++d)
                if (d != 0) lay(x, y + d);
        }
    }

    // electrons on every 20th cell of the shuffled list of laid cells
    void electrons() {
        if (laid_.empty()) return;
        std::shuffle(laid_.begin(), laid_.end(), rng_);
        for (std::size_t i = 0; i < laid_.size(); i += 20) {
            const auto [x, y] = laid_[i];
            at(x, y) = State::electron_head;
            std::vector<std::pair<int, int>> around = {{0, 1}, {1, 0}, {0, -1}, {-1, 0}};
            std::shuffle(around.begin(), around.end(), rng_);
            bool tail = false;
            for (const auto& [dx, dy] : around) {
                if (inside(x + dx, y + dy) && at(x + dx, y + dy) == State::conductor) {
                    at(x + dx, y + dy) = State::electron_tail;
                    tail = true;
                    break;
                }
            }
            if (!tail) at(x, y) = State::conductor;
        }
    }

    int X_, Y_;
    std::vector<State> cells_;
    std::vector<std::pair<int, int>> laid_;
    std::mt19937 rng_;
};

template <typename State>
std::vector<State> circuit_grid(const cellato::run::run_params& params) {
    return circuit_builder<State>((int)params.x_size, (int)params.y_size, static_cast<unsigned>(params.seed)).build();
}

}  // namespace wire

#endif  // WIRE_CIRCUIT_INIT_HPP
