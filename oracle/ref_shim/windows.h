/* Minimal stand-in for the Win32 header the reference includes.
 *
 * TEST INFRASTRUCTURE ONLY: used when compiling the reference's own CPU
 * sources (src/sim/Grid.cpp, src/sim/SimulationCPU.cpp) on Linux so that the
 * reference can verify the oracle restatement and serve as the timed
 * CPU baseline. Nothing in the product links this.
 *
 * The reference uses LARGE_INTEGER / QueryPerformanceCounter /
 * QueryPerformanceFrequency for timers (src/sim/Simulation.h:33-37,
 * src/sim/SimulationCPU.cpp:37-40) and the Win32 min/max macros
 * (src/sim/Grid.cpp:39-40).
 */
#pragma once

#include <chrono>

typedef union ES_LARGE_INTEGER_ {
    long long QuadPart;
} LARGE_INTEGER;

inline int QueryPerformanceCounter(LARGE_INTEGER* c)
{
    c->QuadPart = (long long)std::chrono::duration_cast<std::chrono::nanoseconds>(
                      std::chrono::steady_clock::now().time_since_epoch())
                      .count();
    return 1;
}

inline int QueryPerformanceFrequency(LARGE_INTEGER* f)
{
    f->QuadPart = 1000000000LL;
    return 1;
}

#ifndef max
#define max(a, b) (((a) > (b)) ? (a) : (b))
#endif
#ifndef min
#define min(a, b) (((a) < (b)) ? (a) : (b))
#endif
