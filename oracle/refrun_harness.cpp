/* The reference's whole CPU runner as a C-callable library.
 *
 * TEST INFRASTRUCTURE ONLY. Compiled by oracle/Makefile with the reference's
 * unmodified runner, writers and CPU backend (src/SimulationRunner.cpp,
 * src/Logger.cpp, src/sim/Grid.cpp, src/sim/SimulationCPU.cpp, read in place)
 * into oracle/_ref/libes_refrun.so, so a test can run a .config through the
 * reference's own SimulationRunner::Run (src/SimulationRunner.cpp:32-52) and
 * compare its results folder byte for byte with the B200 runner's.
 *
 * The reference's OpenCL backend (src/sim/SimulationCL.cpp) cannot be built
 * here (no OpenCL headers); the runner only references it for `device gpu`, so
 * its members are defined below as stubs that stop like the reference's error
 * macros do. The test configs select the CPU backend.
 */
#include "src/SimulationRunner.h"

#include <cstdlib>
#include <iostream>

SimulationCL::SimulationCL(int p_particles_per_row, int p_values_per_quadrant, const GridInformation& grid_info,
                           bool p_print_info)
    : Simulation(p_particles_per_row, p_values_per_quadrant, grid_info)
{
    (void)p_print_info;
    std::cout << "The OpenCL backend is not compiled into this harness." << std::endl;
    exit(0);
}

SimulationCL::~SimulationCL() {}

std::vector<Sigma> SimulationCL::ComputeSigmas(const double, const std::vector<double>&, const Grid&, SampleMetrics&)
{
    exit(0);
}

std::vector<IterationResult> SimulationCL::ComputeSigmasWithImages(const double, const std::vector<double>&,
                                                                   const Grid&, SampleMetrics&)
{
    exit(0);
}

extern "C" int refrun(const char* config_path)
{
    InitParameters init;
    init.mode = ProgramMode::Simulation;
    init.config_file = config_path;
    SimulationRunner sr;
    sr.Run(init);
    return 0;
}
