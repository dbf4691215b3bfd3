// Checkpoint files of a chain in the reference's formats: REVIVE (unformatted sequential,
// records of revive, utility_pack.f:1772-1817) and REVCON (CONFIG layout with the final
// coordinates), and the reader of REVIVE (revread, utility_pack.f:1840-1878).
#pragma once
#include <string>
#include <vector>

#include "fmc_inputs.h"

namespace fmc {

struct Revive {
  bool production = false;
  std::vector<int> nummols;        // per FIELD molecule type
  std::vector<double> chainstats;  // 1 + 14 * guest species
  int natms = 0;                   // all atoms, guests and framework
  // per FIELD molecule type: x, y, z of its nummols * numatoms sites
  std::vector<std::vector<double>> x, y, z;
  std::vector<double> energy;  // per guest species, kcal/mol
};

// REVIVE of a chain state: guests from per-species interleaved xyz (molecule-major), the
// framework from the deck.
Revive revive_state(const InputDeck& d, bool production, const std::vector<std::vector<double>>& guest_xyz,
                    const std::vector<double>& chainstats, const std::vector<double>& energy);

// Reads a REVIVE written for the deck's FIELD; 0 or a negative code with a message.
int read_revive(const std::string& path, const InputDeck& d, Revive& r, std::string& err);

// Writes REVIVE records as the reference does (4-byte little-endian record markers, .true.
// as -1 like the shipped example).
int write_revive(const std::string& path, const Revive& r, std::string& err);

// Writes REVCON: the CONFIG title, levcfg 0, imcon and `eng` (the reference writes the last
// move's energy change), the cell, then every atom in condensed order (guests first) with
// Fortran g20.10 coordinates.
int write_revcon(const std::string& path, const InputDeck& d, const Revive& r, double eng, std::string& err);

// Atomic number of a framework atom's mass for the probability cube files, by the mass windows
// of the reference's atmnumber (utility_pack.f:1992-2237); 0 when no window holds the mass.
int atomic_number(double mass);

// Writes one probability plot as a Gaussian cube file (writeprob, utility_pack.f:563-648):
// header, the framework atoms in Bohr, then grid / (cell volume in Bohr^3) / steps, six values
// a line and a new line after every c row.  `grid` is na*nb*nc values, c fastest.
int write_prob_cube(const std::string& path, const InputDeck& d, const double* grid, long long steps,
                    std::string& err);

// Per-species interleaved guest coordinates of a REVIVE.
std::vector<std::vector<double>> revive_guest_xyz(const InputDeck& d, const Revive& r);

}  // namespace fmc
