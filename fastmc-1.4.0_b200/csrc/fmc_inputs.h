// FastMC input deck: CONTROL / FIELD / CONFIG read with the reference's record rules
// (parse_module.f) and directive order (utility_pack.f:176-457 initscan, readinputs.f
// readfield/readconfig/readcontrol).  Errors carry the reference's error codes (error.f).
#pragma once
#include <array>
#include <string>
#include <vector>

namespace fmc {

struct GuestSpecies {
  std::string name;
  int nsite = 0;
  std::vector<std::string> site_name;
  std::vector<double> mass, charge;
  std::vector<double> tx, ty, tz;  // template, centred on the mass COM (readinputs.f:246-268)
  std::vector<int> type;           // 1-based unique atom type (readinputs.f:218-236)
  int nmols = 0;                   // molecules present in CONFIG
  std::vector<double> xyz;         // 3*nmols*nsite, interleaved, molecule-major
};

// One FIELD molecule type in FIELD order (the layout of REVIVE records).
struct MolLayout {
  int guest;      // index into InputDeck::guests, or -1 for a framework type
  int fw_offset;  // framework types: first atom in the condensed framework arrays
  int nummols, numatoms;
};

// One probability plot of a guest species: the sites binned (0 = the centre of mass).
struct ProbPlot {
  int guest = 0;
  std::vector<int> sites;
};

struct InputDeck {
  // initscan
  int imcon = 0, keyfce = 0, kmax[3] = {0, 0, 0};
  double cell[9] = {0};
  double volm = 0, rcut = 0, rvdw = 0, alpha = 0, delr = 0;
  int maxguest = 3000;
  // readfield
  double engunit = 1.0;
  std::vector<std::string> types;  // unique atom types in FIELD order
  std::vector<GuestSpecies> guests;
  // framework atoms in condensed order (all non-guest molecules, FIELD order)
  std::vector<double> fx, fy, fz, fq;
  std::vector<int> ftype, ffrz;
  std::vector<std::string> fname;  // framework site names, condensed order
  std::vector<double> fmass;       // framework site masses, condensed order
  std::vector<MolLayout> mols;     // FIELD molecule types in FIELD order
  std::string title;               // CONFIG's first record, as written
  // probability plots (CONTROL &guest `probability`, `grid spacing`, `grid factors`)
  std::vector<ProbPlot> plots;     // in guest order, then the order given
  double griddim = 0.1;            // gcmc.f:136
  int gridfactor[3] = {1, 1, 1};   // gcmc.f:138
  int ngrid[3] = {0, 0, 0};        // grid cells along a, b, c when plots are requested
  int ntpvdw = 0, maxvdw = 0, mxgrid = 0;
  std::vector<int> ltpvdw, lstvdw;           // [1..maxvdw+1]
  std::vector<std::array<double, 5>> prmvdw;  // [1..maxvdw+1], energies in internal units
  // readcontrol
  double temp = 0;
  int mcsteps = 1, eqsteps = 0, nwind = 100000;
  // numguests.out every nnumg moves (CONTROL `numguests`, else max(1, eqsteps / 1000)) and the
  // guest geometries to his.xyz every |nhis| moves, during production only when nhis > 0
  // (readinputs.f:708-717, 860-866)
  int nnumg = 1, nhis = 0;
  // pressure equilibration during equilibration (CONTROL desorb, adsorb press, adsorb guests,
  // packing fraction, finishment; readinputs.f:749-762): on while despre > 0
  int desorb = 0;
  double despre = 0, packf = 0;
  std::vector<double> adspres, adsguen;
  bool laccsample = false, lspe = false;
  // CONTROL `restart` (readinputs.f:604-608): continue from the REVIVE of this chain's branch
  // directory beside the deck (gcmc.f:353-418; choose_branch in fmc_restart.h)
  bool lrestart = false;
  std::vector<double> press;  // Pa, per guest
  std::vector<std::array<double, 9>> movefreq;  // ins,del,dis,jmp,flx,swp,tra,rot,mjp (raw)
  std::vector<double> disp_ratio, tran_ratio;
  double rota_ratio = 0.5;
};

// Reads dir/{CONTROL,FIELD,CONFIG}.  Returns 0, or the reference's error code (>0); `err`
// receives a message.  Directives outside this path are rejected with a negative code.
int read_input_deck(const std::string& dir, InputDeck& deck, std::string& err);

// A deck whose arrays a caller filled in memory (the state the reference's module arrays hold
// after readfield / readconfig / readcontrol): checks the cell against its image convention and
// the cut-off against the half-cell width as readconfig does, then derives the volume, mxgrid,
// the vdW pair-table map (undefined pairs -> the zero table) and the numguests interval.
// Expects types, framework and guest arrays, ntpvdw with ltpvdw / prmvdw [ntpvdw+1] and lstvdw
// [ntypes*(ntypes+1)/2+1] (0 = no line), cell, imcon, alpha, kmax, rcut and the control fields.
int finish_deck_from_arrays(InputDeck& d, std::string& err);

}  // namespace fmc
