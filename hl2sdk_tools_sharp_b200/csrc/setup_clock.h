// setup_clock.h -- wall-clock phases of the host-side set-up (the world
// and bounce uploads).  With the environment variable VRAD_SETUP_TIMES set,
// each mark() prints "[vrad setup] <entry> <phase> <ms>" to stderr; without
// it a mark costs one branch.
#pragma once

#include <chrono>
#include <cstdio>
#include <cstdlib>

namespace vrad {

class SetupClock {
public:
    explicit SetupClock(const char *entry)
        : entry_(entry), on_(std::getenv("VRAD_SETUP_TIMES") != nullptr), t_(Clock::now()) {}

    void mark(const char *phase) {
        if (!on_) return;
        const Clock::time_point t = Clock::now();
        std::fprintf(stderr, "[vrad setup] %s %s %.2f ms\n", entry_, phase,
                     std::chrono::duration<double, std::milli>(t - t_).count());
        t_ = t;
    }

private:
    using Clock = std::chrono::steady_clock;
    const char *entry_;
    bool on_;
    Clock::time_point t_;
};

}  // namespace vrad
