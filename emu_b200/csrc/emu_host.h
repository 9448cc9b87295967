// emu_host.h -- host-only helpers of the C ABI (no CUDA): physical constants,
// parameter validation, the vacuum mass matrix, fixed-point scales, and the
// AMReX plotfile / particle checkpoint writer.
#pragma once

#include <string>
#include <vector>

#include "emu_b200.h"
#include "emu_init_record.h"

namespace emu_host {

// Source/Constants.H:6-26, evaluated in the same operation order
double c2();
double c4();
double hbarc();
double gf();

bool validate(const emu_params& p, std::string& why);

// message returned by emu_last_error(NULL, ...)
void set_error(const std::string& msg);

// flavour-basis mass-squared matrix in Hermitian component order for nu
// (m2[0]) and nubar (m2[1], conjugated), generate_code.py:174-255
void vacuum_m2(const emu_params& p, double m2[2][9]);

// int64 fixed-point scales for the mixed deposit: contribution * scale is an
// integer with |sum over any cell| < 2^62 (bound: total N per species)
bool fixed_point_scales(const emu_params& p, const double* records, long long n, double scale[2],
                        double unscale[2], std::string& why);
// the same from per-species sums and maxima of |N| (summed / maxed over the
// ranks of a sharded run first)
void weight_totals(const emu_params& p, const double* records, long long n, double total[2], double mx[2]);
bool fixed_point_scales_from(const double totals[2], const double maxima[2], double scale[2], double unscale[2],
                             std::string& why);

// Vvac_max (FlavoredNeutrinoContainerInit.cpp:657-660) from the smallest
// particle energy
double vvac_from_pupt_min(const emu_params& p, double pupt_min);

// inputs of the initial-particle generator (emu_init_record.h); total =
// particle count
bool make_init_spec(const emu_params& p, emu_init::InitSpec& s, std::vector<double>& dirs, long long& total,
                    std::string& why);

bool write_plotfile(const emu_params& p, const char* dir, double time, int step, const double* mesh,
                    const double* records, long long n, std::string& why);

}  // namespace emu_host
