// setup_clock.h -- wall-clock phases of the host-side set-up (the world
// and bounce uploads).  With the environment variable VRAD_SETUP_TIMES set,
// each mark() prints "[vrad setup] <entry> <phase> <ms> (cpu <ms>)" to
// stderr, the second figure the process's CPU time over the phase (all
// threads); without it a mark costs one branch.
#pragma once

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <ctime>

namespace vrad {

class SetupClock {
public:
    explicit SetupClock(const char *entry)
        : entry_(entry), on_(std::getenv("VRAD_SETUP_TIMES") != nullptr), t_(Clock::now()), cpu_(cpu_ms()) {}

    void mark(const char *phase) {
        if (!on_) return;
        const Clock::time_point t = Clock::now();
        const double c = cpu_ms();
        std::fprintf(stderr, "[vrad setup] %s %s %.2f ms (cpu %.1f ms)\n", entry_, phase,
                     std::chrono::duration<double, std::milli>(t - t_).count(), c - cpu_);
        t_ = t;
        cpu_ = c;
    }

private:
    using Clock = std::chrono::steady_clock;
    static double cpu_ms() {
        timespec ts;
        clock_gettime(CLOCK_PROCESS_CPUTIME_ID, &ts);
        return (double)ts.tv_sec * 1e3 + (double)ts.tv_nsec * 1e-6;
    }
    const char *entry_;
    bool on_;
    Clock::time_point t_;
    double cpu_;
};

}  // namespace vrad
