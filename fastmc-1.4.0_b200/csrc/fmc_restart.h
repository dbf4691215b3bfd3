// Checkpoint files of a chain in the reference's formats: REVIVE (unformatted sequential,
// records of revive, utility_pack.f:1772-1817) and REVCON (CONFIG layout with the final
// coordinates), and the reader of REVIVE (revread, utility_pack.f:1840-1878).
#pragma once
#include <string>
#include <vector>

#include "fmc_common.h"
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

// The final statistics of the reference's report (gcmc.f:1960-2037), in the chainstats layout:
// out[0] production moves; per species g at 1 + 14 g: <N>, <E>, <EN>, <N^2>, <E^2>, the sixth
// average, then the errors of N, E, EN, N^2, E^2, Q_st, Cv and the sixth.  Up to 500,000
// production moves the averages and errors come from 5 blocks of the stored samples (gasmol,
// gaseng; each block sums the nwind + 1 samples of an inclusive slice and divides by nwind, as
// the reference does); beyond, from the averaging windows closed during the run.
void final_stats(int ng, double temp, const double* chainstats, const WindowStats& W, const double* gasmol,
                 const double* gaseng, double* out);

// Window state as a flat array: avcount, rollcount, then sum[8 ng], var[8 ng], avg[8 ng] and
// seltot[ng ng] (species-major).
void window_stats_out(const WindowStats& W, int ng, double* out);

// The reference's per-node report block (gcmc.f:2052-2117) for one chain: every species'
// averages, production moves, Q_st and Cv with their errors, then the selectivities.
int write_report(const std::string& path, const InputDeck& d, const double* final_cs, const WindowStats& W,
                 double temp, std::string& err);

// Where node `idnode` (0-based) of a job whose CONTROL says `restart` takes its state from
// (gcmc.f:353-394): prevnodes counts the entries of `workdir` whose names contain "branch" (revscan,
// utility_pack.f:1819-1839, lists the working directory); with none the node starts from the
// CONFIG; node idnode < prevnodes reads branch{idnode+1}/REVIVE, a node beyond them
// branch{mod(idnode+1, prevnodes)+1}/REVIVE; a missing REVIVE also means the CONFIG (revread's
// status-old test, utility_pack.f:1855-1860).  The node's own output directory is
// branch{idnode+1} either way.
struct BranchChoice {
  int prevnodes = 0;
  std::string outdir;  // workdir/branchNN of this node
  std::string revive;  // the REVIVE to read, or empty: start from the CONFIG
};
// 0, or -1 with a message for a node index beyond the reference's two-digit branch names.
int choose_branch(const std::string& workdir, int idnode, BranchChoice& out, std::string& err);

// Per-species interleaved guest coordinates of a REVIVE.
std::vector<std::vector<double>> revive_guest_xyz(const InputDeck& d, const Revive& r);

}  // namespace fmc
