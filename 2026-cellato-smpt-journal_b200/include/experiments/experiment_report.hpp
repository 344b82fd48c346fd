// Experiment report: per-round times and checksums, CSV line (same columns as
// the reference include/experiments/experiment_report.hpp:82-127: the
// run_params columns, then average_time_ms, average_time_per_cell_ps,
// std_time_ms, rounds_had_same_checksums, checksum).
#ifndef CELLATO_EXPERIMENT_REPORT_HPP
#define CELLATO_EXPERIMENT_REPORT_HPP

#include <cmath>
#include <iostream>
#include <string>
#include <vector>

#include "./run_params.hpp"

namespace cellato::run {

struct experiment_report {
    run_params params;
    std::vector<double> execution_times_ms;
    std::vector<std::string> checksums;

    static std::string csv_header() {
        return run_params::csv_header() +
               ",average_time_ms,average_time_per_cell_ps,std_time_ms,rounds_had_same_checksums,checksum";
    }
    std::string csv_line() const {
        return params.csv_line() + "," + std::to_string(average_time_ms()) + "," +
               std::to_string(average_time_per_cell_ps()) + "," + std::to_string(std_time_ms()) + "," +
               (rounds_had_same_checksums() ? "true" : "false") + "," + (checksums.empty() ? "" : checksums[0]);
    }
    double average_time_ms() const {
        double s = 0;
        for (double t : execution_times_ms) s += t;
        return execution_times_ms.empty() ? 0 : s / execution_times_ms.size();
    }
    double std_time_ms() const {
        const double m = average_time_ms();
        double s = 0;
        for (double t : execution_times_ms) s += (t - m) * (t - m);
        return execution_times_ms.empty() ? 0 : std::sqrt(s / execution_times_ms.size());
    }
    bool rounds_had_same_checksums() const {
        for (const auto& c : checksums)
            if (c != checksums[0]) return false;
        return true;
    }
    // picoseconds per cell update
    double average_time_per_cell_ps() const {
        if (params.x_size == 0 || params.y_size == 0 || params.steps == 0) return 0;
        return average_time_ms() * 1e9 / (double(params.x_size) * params.y_size) / params.steps;
    }
    void pretty_print(std::ostream& os) const {
        os << "Grid " << params.x_size << " x " << params.y_size << ", " << params.steps << " steps, "
           << execution_times_ms.size() << " rounds: " << average_time_ms() << " ms (std " << std_time_ms()
           << "), " << average_time_per_cell_ps() << " ps/cell, "
           << (rounds_had_same_checksums() ? "consistent" : "INCONSISTENT") << " checksum "
           << (checksums.empty() ? "" : checksums[0]) << "\n";
    }
};

}  // namespace cellato::run

#endif
