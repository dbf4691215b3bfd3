// Host-side system description built once per input deck: interpolation tables, the
// k-vector table, the long-range-correction terms, per-guest constants and the framework
// voxel neighbour lists that replace the reference's per-trial brute-force list
// (guestlistgen, utility_pack.f:3113-3177).
#pragma once
#include <string>
#include <vector>

#include "fmc_common.h"
#include "fmc_inputs.h"

namespace fmc {

struct HostSystem {
  InputDeck deck;
  CellGeom cell;
  double rcut = 0, alpha = 0, engunit = 0, beta = 0, statvolm = 0;
  int mxgrid = 0;
  double drewd = 0, dlrpot = 0;
  std::vector<double> erc;    // [mxgrid+1], erc[0] := erc[1]
  int ntables = 0;            // vdW tables incl. the zero table
  std::vector<double> vvv;    // [ntables+1][mxgrid+1], row 0 unused
  int ntypes = 0;
  std::vector<int> pair_row;  // [(ntypes+1)^2] -> vvv row, -1 = pair skipped
  // reciprocal space
  int K = 0;
  std::vector<int> kl, km, kn;  // reference half-space enumeration order (ewald.f:139-331)
  std::vector<double> akk;
  double recip_pref = 0;  // 2*(2 pi/V)*r4pie0/epsq (lconsw) or (2 pi/V)*r4pie0/epsq
  // long-range correction (lrcorrect / gstlrcorrect, vdw_terms.f:500-745)
  std::vector<double> steadd;  // [ntab+1]
  bool lrc_on = false;
  // guests
  std::vector<double> engsic;    // self term per guest type (ewald.f:87-93)
  std::vector<double> ewald3en;  // intramolecular correction per guest type (gcmc.f:529-552)
  // move thresholds (cumulative, gcmc.f:282-331) per guest
  std::vector<std::array<double, 9>> mvcum;
  // framework (condensed order)
  int nf = 0;
  std::vector<double> fx, fy, fz, fq;
  std::vector<int> ftype, ffrz;
  // voxel neighbour lists: every framework atom whose minimum-image distance to the voxel
  // centre is below rcut + the voxel's circumradius (built on the device by upload_system;
  // build_host_voxels fills the host copies for inspection)
  int nvox[3] = {1, 1, 1};
  double vox_lim2 = 0;
  long long vox_entries = 0;
  std::vector<int> vox_off, vox_atoms;
};

// Host construction of the voxel lists (the device builds the same lists in upload_system).
void build_host_voxels(HostSystem& sys);

// Builds everything above from a deck.  Returns 0 or an error code; fills err.
int build_host_system(const InputDeck& deck, HostSystem& sys, std::string& err, double voxel_edge = 2.0);

// A&S 7.1.26 erf-based intramolecular correction of one pair (ewald3, ewald.f:697-758).
double ewald3_pair(double alpha, double chgprd, double rrr);

// Tail correction of the whole system from per-type counts (gstlrcorrect).
double lrc_energy(const HostSystem& s, const std::vector<int>& numtyp, const std::vector<int>& numfrz);

}  // namespace fmc
