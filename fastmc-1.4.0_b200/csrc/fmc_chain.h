// One GCMC chain on one GPU: device-resident system + S(k) + guest sites, and the host move
// loop of the plain path (gcmc.f:589-1380 restated, energies from fmc_kernels.cu).
#pragma once
#include <cstdio>
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "fmc_kernels.h"
#include "fmc_system.h"

namespace fmc {

// Per-move record, identical in layout to fmc_move_record of the C ABI.
struct MoveRecord {
  int32_t step, iguest, mtype, randchoice, accepted, nmols_after, pad0, pad1;
  double ewld1, ewld2, ewld3, vdw, delrc, estep, rande, energy_after;
};

// Device copy of one system (immutable arrays) -- shared by chains of the same framework.
struct DeviceSystem {
  DevSystem view{};
  std::vector<void*> allocations;
  int device = 0;
  long long vox_entries = 0;
  ~DeviceSystem();
};

int upload_system(const HostSystem& h, DeviceSystem& d, std::string& err);

struct Species {
  int nsite = 0, seg_off = 0, cap_sites = 0, nmol = 0;
  std::vector<double> xyz;  // 3*nmol*nsite, molecule-major (framwkxxx of the reference)
};

// Host part of opening a chain: reads the deck, checks what the GPU path supports and
// builds the host tables.  Thread-safe (no device calls).
// voxel_edge: target edge (A) of the voxels whose neighbour lists the kernels read.
int prepare_system(const std::string& dir, HostSystem& sys, std::string& err, double voxel_edge = 2.0);

class Chain {
 public:
  HostSystem sys;
  DeviceSystem dsys;
  int device = 0;
  cudaStream_t st = nullptr;
  // device chain state
  double2* sk = nullptr;
  double2* sk_new = nullptr;
  double2* sk_save = nullptr;  // S(k) before a multi-jump, restored if it is rejected
  double4* gsite = nullptr;
  int* gtype = nullptr;
  int gcap = 0;
  PassScratch W{};
  double* recip_scratch = nullptr;
  double* recip_parts = nullptr;
  size_t recip_scratch_n = 0;
  double4* all_atoms = nullptr;
  int all_cap = 0;
  // host mirror
  std::vector<Species> sp;
  int totatm = 0, framatm = 0;
  std::vector<int> numtyp, numfrz;
  double elrc = 0;
  std::vector<double> energy, delE;
  // set-up energies
  double spenergy = 0, dlpeng = 0, ewald1sum = 0;
  // move-loop control (gcmc.f:320-588)
  Duni rng{};
  int gcmccount = 0;
  std::vector<double> delrdisp, tran_delr;
  std::vector<int> accept_disp, disp_count, accept_tran, tran_count;
  int accept_rota = 0, rota_count = 0, accept_ins = 0, accept_del = 0, ins_count = 0, del_count = 0;
  double rotangle = kPi / 3.0, rota_rotangle = kPi / 3.0;
  bool production = false, lgchk = true;
  long long prodcount = 0;
  bool tick_tock[5] = {false, false, false, false, false};
  std::vector<double> chainstats;  // 1 + 14*ntpguest, <N>,<E>,<EN>,<N^2>,<E^2> rolling
  // partial pressures (Pa) the acceptance uses; the pressure equilibration changes them while
  // despre > 0 (gcmc.f:637-696)
  std::vector<double> gstpress;
  double despre = 0, presrate = 0;
  // launch accounting and optional CUDA-event timing of the pass kernel
  long long passes = 0, commits = 0;
  double pass_seq = 0.0;  // sequence number the pass kernel echoes next to its energies
  bool profile = false;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  double pass_ms = 0.0;
  long long pass_timed = 0;
  // numguests.out and his.xyz (gcmc.f:418-450), open while a caller asked for them
  std::vector<std::FILE*> numg_f, his_f;

  ~Chain();
  // Opens the trajectory files in `dir` (numguestsNN.out / hisNN.xyz per species for
  // mixtures); an empty dir closes them.
  int open_outputs(const std::string& dir, std::string& err);
  void close_outputs();
  int open(const std::string& dir, const int seed[4], int device, std::string& err, double voxel_edge = 2.0);
  // open from a system already built on the host by prepare_system (the device part only)
  int open_prepared(HostSystem&& prepared, const int seed[4], int device, std::string& err);
  GuestView guest_view() const;
  // Energies of one trial pass.  old_xyz/new_xyz are interleaved xyz of the molecule's sites.
  int pass(int move, int g, int mol, const double* old_xyz, const double* new_xyz, double out[3]);
  // An accepted move: S(k) <- S_new by exchanging the two buffers, and the guest-site update
  // left pending for the next pass to read through and write (no launch of its own); a second
  // update before the next pass, or one of more than kMaxPendSites sites, is written at once.
  int commit(int move, int g, int mol, const double* new_xyz);
  // Hands the pending guest-site update to a pass about to launch (or marks none).
  void take_pending(PassArgs& A);
  // Writes the pending guest-site update now (before anything else reads the device sites).
  int flush_commit();
  PendingCommit pend{};
  bool pend_live = false;
  // Resident pass kernel (fmc_pass_server_kernel on its own stream): passes of up to
  // kSmallPassSites sites go through its mailbox instead of a launch each.  Any other device
  // work on the chain stops it first (stop_server); the next pass starts it again.
  bool use_server = false;  // off by default: opt in with fmc_chain_resident
  bool srv_live = false;
  bool st_dirty = false;           // work queued on `st` since the last synchronisation
  cudaStream_t srv_st = nullptr;
  PassMailbox* mb = nullptr;       // pinned
  PassServerFlags* d_fl = nullptr;
  PassServerFlags* h_fl = nullptr; // pinned staging of the flags a launch starts from
  int* srv_words = nullptr;        // pinned: [0] ended, [1] reason a wait ran out
  double pass_seq_done = 0.0;      // last pass whose result the host has read
  long long srv_launches = 0, srv_passes = 0;
  int start_server();
  int stop_server();
  int pass_resident(const PassArgs& A, double out[3]);
  int full_recip(double* e_recip_plus_self);  // S(k) over all current atoms (ewald1)
  int single_point();
  int step(MoveRecord* rec);
  int set_guests(int g, int nmol, const double* xyz);  // replace species g (condense equivalent)
  // Restart from a REVIVE (gcmc.f:353-418, revread): the stored guests, a fresh single point,
  // every species' energy set to it, the production flag and chain statistics.
  int restart(const struct Revive& r, std::string& err);
  int last_guest = 0;  // species of the last move (the reference's REVCON energy is its delE)
  bool last_accepted = false;  // flex / swap moves report the previous move's flag
  WindowStats win;                      // the reference's averaging windows
  std::vector<double> gasmol, gaseng;   // first production samples of N and E per species
  int jump_count = 0, accept_jump = 0;
  // probability plots (storeprob): one grid per plot of the deck, weights summed in FP64
  std::vector<std::vector<double>> prob;
  void store_prob();
  int sync_error(cudaError_t e, std::string* err = nullptr);
};

}  // namespace fmc
