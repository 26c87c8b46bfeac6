// es_host_math.h - host-side FP64 set-up arithmetic shared by the per-pass
// context (es_context.cu) and the batched path (es_batch.cu).
//
// Everything here must agree with the reference's CPU code bit for bit, so the
// translation units that include it are compiled for the host without FMA
// contraction (-Xcompiler -ffp-contract=off) and use the host libm.
#pragma once

#include "es_cuda.h"
#include "es_internal.h"

#include <cmath>

namespace es {
namespace host {

// src/sim/es/constants.h:23-35
constexpr double kM0 = 9.10938188e-31;
constexpr double kM = (5.0 * kM0);
constexpr double kE = 1.60217646e-19;
constexpr double kHBAR = 1.05457148e-34;
constexpr double kC1 = 1.15e-9;
constexpr double kKB = 1.380649e-23;
constexpr double kPI = 3.141592653589793238463;
constexpr double kPI2 = 6.283185307179586;
constexpr double kHALF_PI = 1.570796326794896619231;

inline double smod(double a, double b) { return a - b * std::floor(a / b); }

// SimpsonWeight, src/sim/es/util.h:24-28
inline double simpson_weight(int i, int dim)
{
    const double main_multiplier = (i % 2 == 0) ? 2.0 : 4.0;
    const bool is_edge = (i == 0) || i == (dim - 1);
    return is_edge ? 1.0 : main_multiplier;
}

// Angular speed, SimulationCPU::ComputeLifetimes, src/sim/SimulationCPU.cpp:107
inline double angular_speed(double magnetic_field) { return kE * magnetic_field / kM; }

// GetTau, src/sim/Simulation.h:90
inline double get_tau(bool coherent, double tau, double temperature)
{
    return coherent ? tau : kHBAR / (kKB * temperature);
}

// GetSigmaIntegrandFactor with SigmaFactor inlined, src/sim/Simulation.h:69-76,88
inline double integrand_factor(double particle_speed, int positions_per_row, double phi_integrand_factor, double w,
                               double tau)
{
    const double kf = kM * particle_speed / kHBAR;
    double outside = (kE * kE * kf * kf) / (2.0 * kPI * kPI * kM * kC1);
    const double wct = w * tau;
    outside *= tau / (1.0 + wct * wct);
    return std::pow(1.0 / (3.0 * (positions_per_row - 1)), 2) * phi_integrand_factor * outside * 1e-8;
}

// Whether a grid's walks are long enough for the split lifetime kernel to
// leave the winners' FP64 times to its finish kernel: the straight-line mean
// free path through its disks, L / (disks filed per cell x 2 r_i), at least
// half a cell. Around one cell or more (5e15 m^-2, r_i 2 nm, 49 nm cells:
// 0.87) walks end after differing numbers of cell steps and the split finish
// pays (5% per pass on B200); well below (1e16 m^-2, r_i 5 nm, 35 nm cells:
// ~0.2) nearly every walk ends in its first cell and it measured 9-10%
// slower than the finish inside the walk.
inline bool long_walks(int64_t n_indexed, int cells_per_row, double cell_size, double impurity_radius)
{
    const double cells = (double)cells_per_row * (double)cells_per_row;
    const double per_cell = cells > 0.0 ? (double)n_indexed / cells : 0.0;
    if (!(per_cell > 0.0) || !(impurity_radius > 0.0)) return true;
    return cell_size / (per_cell * 2.0 * impurity_radius) >= 0.5;
}

// Upper bound on the cell steps of one orbit: a full circle crosses at most
// 4 * ceil(2 pi r / cell) + a few cell edges. Exceeding it is reported.
inline int walk_cap_for(double radius, double cell)
{
    const double steps = 4.0 * std::ceil(kPI2 * radius / cell) + 16.0;
    return steps > 2.0e9 ? 2000000000 : (int)steps;
}

// The split walk's FP32 constants of a pass (trace_split in es_orbit_split.cuh
// uses them; they depend on the orbit radius, the impurity radius and the cell
// size only). The same IEEE operations as the device expressions they replace:
// FP64 products rounded to FP32 once, FP32 products rounded after each step.
inline void split_constants(LifetimeLaunch& L)
{
    const double r64 = L.radius, ir64 = L.imp_radius;
    L.sc_r = (float)r64;
    L.sc_inv_r = (float)(1.0 / r64);
    L.sc_ir = (float)ir64;
    L.sc_lo2 = (float)((r64 - ir64) * (r64 - ir64));
    L.sc_hi2 = (float)((r64 + ir64) * (r64 + ir64));
    const float t = 2e-6f * L.sc_r;
    L.sc_eps2 = t * L.sc_r;
    L.sc_band_d = 0.02f * L.sc_ir;
    L.sc_inv4r = 0.25f * L.sc_inv_r;
    L.sc_tangent_tol = (float)((0.01 * L.cell_size * L.cell_size) * (double)L.sc_inv_r + 2e-7 * L.cell_size);
    // M = ceil(2^64 / d): for n, d < 2^32, (n M) >> 64 = floor(n / d), since
    // n M / 2^64 exceeds n / d by less than 2^-32 < 1 / d
    L.inv_phase = L.n_phase > 0 ? UINT64_MAX / (uint64_t)L.n_phase + 1 : 0;
    L.inv_dim = L.dim > 0 ? UINT64_MAX / (uint64_t)L.dim + 1 : 0;
}

// Sector constants of Simulation::InitSample (src/sim/Simulation.h:111-126).
struct Sector {
    double area, phi_integrand_factor, phi_start, phi_step;
};

inline Sector sector(double alpha, int ppq, bool coherent)
{
    const double base_area = alpha * 2.0;
    Sector s;
    s.area = !coherent ? base_area : (kHALF_PI - base_area);
    s.phi_integrand_factor = s.area / ((ppq - 1) * 3.0);
    s.phi_start = (!coherent ? -alpha : alpha);
    s.phi_step = s.area / (ppq - 1);
    return s;
}

// Phase tables of one sector (4 * ppq entries, [q][p]): CreateParticle's
// per-phase constants (src/sim/es/lifetime.h:39-45), GetBoundTime's angle
// (src/sim/es/details.h:219-228) and ApplySigma's cos/sin and weight
// (src/sim/SimulationCPU.cpp:186-192,218).
inline void phase_tables(const Sector& sec, int ppq, double particle_speed, double alpha, bool clockwise,
                         PhaseOrbit* po, PhaseSigma* psg)
{
    for (int q = 0; q < 4; q++) {
        for (int p = 0; p < ppq; p++) {
            const int v = q * ppq + p;
            const double phi = sec.phi_start + q * kHALF_PI + p * sec.phi_step;
            PhaseOrbit& o = po[v];
            o.phi = phi;
            o.vel_x = std::cos(phi) * particle_speed;
            o.vel_y = std::sin(phi) * particle_speed;
            const double remaining = smod(phi + alpha, kHALF_PI);
            o.bound_dphi = clockwise ? remaining : (2.0 * alpha - remaining);
            PhaseSigma& g = psg[v];
            g.phi = phi;
            g.cos_phi = std::cos(phi);
            g.sin_phi = std::sin(phi);
            g.weight = simpson_weight(p, ppq);
        }
    }
}

}  // namespace host
}  // namespace es
