// Batched path: many independent GCMC chains advanced by one persistent kernel, one CTA per
// chain, the whole move loop of gcmc.f:589-1380 on the device.  Chains that share a framework
// deck (same FIELD / CONFIG / cut-offs / Ewald parameters) share one device system.
#pragma once
#include <functional>
#include <cuda_runtime.h>

#include <memory>
#include <string>
#include <vector>

#include "fmc_chain.h"

namespace fmc {

constexpr int kBatchMaxSites = 16;  // sites per guest species on the batched path
constexpr int kBatchMaxTypes = 16;  // unique atom types
constexpr int kBatchMaxTab = kBatchMaxTypes * (kBatchMaxTypes + 1) / 2;
// Tile shapes of the batched kernel the autotuner chooses among: threads per chain (CTA size),
// k-vectors each thread takes per trip of the reciprocal loop (ewald.f:145-331) and neighbour
// candidates per trip of the real-space loop (ewald.f:656-690, vdw_terms.f:455-495).  Tile 0
// is the default.  Within one thread-count the tiles give bit-identical results (each thread
// sums its k-vectors and candidates in the same order); another thread count sums in another
// order.  One chain per CTA throughout: two chains share an SM as two CTAs.
struct BatchTile {
  int threads, kvec_per_trip, cand_per_trip;
};
constexpr int kNumBatchTiles = 12;
constexpr BatchTile kBatchTiles[kNumBatchTiles] = {
    {256, 1, 1}, {256, 2, 1}, {256, 1, 2}, {256, 2, 2}, {128, 1, 1}, {128, 2, 1},
    {128, 1, 2}, {128, 2, 2}, {384, 1, 1}, {384, 2, 1}, {384, 1, 2}, {384, 2, 2}};
constexpr int kMaxPlots = 8;      // probability plots per system
constexpr int kMaxPlotSites = 8;  // sites per plot (0 = centre of mass)

struct SpeciesConst {
  int nsite;
  double tx[kBatchMaxSites], ty[kBatchMaxSites], tz[kBatchMaxSites];
  double q[kBatchMaxSites], mass[kBatchMaxSites];
  int type[kBatchMaxSites];
  double engsic, ewald3en;
};

// Per-system constants (device memory, read-only during a launch).
struct SysConst {
  DevSystem S;
  int nspecies, ntypes, lrc_on;
  SpeciesConst sp[kMaxGuestTypes];
  double steadd[kBatchMaxTab + 1];
  int numfrz[kBatchMaxTypes + 1];
  double engunit, volm, statvolm;
  // probability plots (storeprob): grid cells per axis, and per plot its species and sites
  int nplots, ngrid[3];
  int plot_guest[kMaxPlots], plot_nsite[kMaxPlots], plot_site[kMaxPlots][kMaxPlotSites];
};

// Per-chain parameters and mutable state (device memory).
struct ChainDev {
  int sys;
  int status;  // 0 ok; 75 guest capacity exhausted (the reference's error 75)
  int active;  // 0: an empty serving slot (the launch skips it)
  long long budget;  // total moves this chain is to run (0: unlimited)
  // parameters (CONTROL)
  double temp, beta, press[kMaxGuestTypes], mvcum[kMaxGuestTypes][9];
  double disp_ratio[kMaxGuestTypes], tran_ratio[kMaxGuestTypes], rota_ratio;
  int maxguest, mcsteps, eqsteps, laccsample;
  // move-loop state
  Duni rng;
  int gcmccount, totatm, framatm;
  int nmol[kMaxGuestTypes];
  int numtyp[kBatchMaxTypes + 1];
  int disp_count[kMaxGuestTypes], accept_disp[kMaxGuestTypes];
  int tran_count[kMaxGuestTypes], accept_tran[kMaxGuestTypes];
  int rota_count, accept_rota, ins_count, del_count, accept_ins, accept_del;
  int jump_count, accept_jump, last_accepted;
  double delrdisp[kMaxGuestTypes], tran_delr[kMaxGuestTypes], rotangle, rota_rotangle;
  double elrc, energy[kMaxGuestTypes];
  double last_dE;  // energy change of the last move if accepted, else 0 (the reference's delE)
  int production, lgchk, tick[5];
  long long prodcount;
  // pressure equilibration (gcmc.f:637-696, 1796-1808), on while despre > 0; press[] changes
  double despre, packf, presrate, adspres[kMaxGuestTypes], adsguen[kMaxGuestTypes];
  double stats[kMaxGuestTypes][6];  // rolling <N>, <E>, <EN>, <N^2>, <E^2>, <exp(-dE/kT)> of insertions
  WindowStats win;                  // the reference's averaging windows
  int nwind;                        // production samples per window (CONTROL `averaging window`)
  double* gasmol;                   // first production samples of N and E per species
  double* gaseng;                   // ([nspecies * 500000 + 1]; null: not recorded)
  long long moves_done;
  // SM clock cycles spent per phase when the launch is profiled: begin (thread 0), phase
  // tables, k-space + real space + reduction, end (thread 0), commit
  long long prof[12];
  // buffers
  double2* sk;
  double4* gsite;
  int* gtype;
  int seg_off[kMaxGuestTypes], seg_cap[kMaxGuestTypes];
  // probability plots: nplots grids of weights in fixed point (units of 2^-32), summed with
  // integer atomics so the totals do not depend on the order of the adds
  unsigned long long* prob;
};

struct BatchLaunch {
  ChainDev* chains;
  const SysConst* systems;
  int nchains, moves;
  MoveRecord* trace;  // [nchains][moves] or null
  int kmax_smem;      // largest K in the batch rounded up to a multiple of 4 (smem sizing)
  int profile;        // accumulate per-phase clock counters into ChainDev::prof
  const int* order;   // optional [nchains]: the chain each CTA runs (placement only: a chain's result
                      // does not depend on its CTA)
  long long* timing;  // optional [nchains][3] per chain: its CTA's start and end (%globaltimer, ns), its SM
  int retire_finished;  // a chain that ends its budget, its deck's cycles or on an error marks itself
                        // inactive, so that a launch queued behind this one skips it (serving)
  int tile;             // index into kBatchTiles (profiling runs tile 0 only)
};

cudaError_t launch_batch(const BatchLaunch& L, int smem_bytes, int tab_stride, cudaStream_t st);
int batch_smem_bytes(int kmax_K, int tab_sites, int tab_stride);
cudaError_t configure_batch_kernel(int smem_bytes);

using DevAllocFn = std::function<cudaError_t(void**, size_t)>;
int fill_sysconst(const HostSystem& H, const DevSystem& S, SysConst& Y, int* tab_sites, std::string& err);
int make_sysconst(const Chain& ch, SysConst& Y, std::vector<void*>& allocations, int* tab_sites, std::string& err);
// record_samples: allocate the first production samples of N and E (gasmol / gaseng, 16 MB a
// species) that the final report's blocked errors need up to 500,000 production moves.
// Device bytes init_chain_state allocates for a chain (before alignment).
size_t chain_state_bytes(const InputDeck& d, const HostSystem& H, bool record_samples);
int init_chain_state(const InputDeck& d, const HostSystem& H, const double2* sk_src, double energy0, int sys,
                     const int* seed, ChainDev& C, const DevAllocFn& alloc, cudaStream_t st, std::string& err,
                     bool record_samples);
int init_chain(const InputDeck& d, const Chain& ch, int sys, const int* seed, ChainDev& C,
               std::vector<void*>& allocations, cudaStream_t st, std::string& err);

// Device memory of one serving slot.  Every allocation comes from a memory pool on the
// slot's stream, so admitting and retiring slots needs no device-wide synchronisation.
struct SlotMemory {
  cudaStream_t st = nullptr;
  cudaMemPool_t pool = nullptr;
  std::vector<void*> ptrs;
  size_t bytes = 0;
  // one pool allocation that later alloc() calls carve (256-byte aligned) until it is used up;
  // a slot's buffers then cost one allocation call instead of one each
  unsigned char* arena = nullptr;
  size_t arena_cap = 0, arena_used = 0;
  cudaError_t reserve(size_t n);
  cudaError_t alloc(void** p, size_t n);
  void release();  // stream-ordered frees of every allocation
};

// Pinned host staging for slot uploads: a bump allocator over one pinned buffer; its owner
// resets `used` once the stream that reads the staged bytes has drained.
struct Staging {
  unsigned char* base = nullptr;
  size_t cap = 0, used = 0;
  void* take(size_t n);  // 256-byte aligned; nullptr when the buffer is full
};

// Pinned bytes build_slot stages for a system.
size_t slot_staging_bytes(const HostSystem& h);
// Voxel-list entries of a system estimated from its framework density (+15% and 4096).
long long slot_voxel_capacity(const HostSystem& h);

// A slot that starts with guests instead of the empty framework: the guests the deck preloads
// (FIELD NUMMOLS > 0), or a REVIVE's (CONTROL `restart`), with the S(k) of every atom and the
// single-point energy (gcmc.f:500-556) that a chain opened on the same deck computed, all in
// host memory.  From a REVIVE also its production flag and chain statistics (gcmc.f:396-409).
struct SlotStart {
  std::vector<double2> sk;                  // K entries
  double spenergy = 0.0;                    // kcal/mol, every species' starting energy
  std::vector<int> nmol;                    // per species
  std::vector<std::vector<double4>> sites;  // per species, nmol * nsite sites (x, y, z, q)
  std::vector<std::vector<int>> types;      // per species, their atom types
  bool from_revive = false;
  bool production = false;
  std::vector<double> chainstats;           // 1 + 14 * species
};

// A serving slot built from a prepared host system: the device system (framework, voxel lists,
// tables), the framework S(k), the per-system constants and an empty chain (or one starting
// from `start`, whose host arrays the call copies before it returns), all enqueued on
// mem.st without waiting (one staged host-to-device copy; voxel lists sized by vox_cap entries,
// the exact count copied to *vox_total, pinned, for the caller to check once mem.st has
// drained: a total above vox_cap means the lists are cut and the slot must be rebuilt with
// vox_cap = total).
int build_slot(const HostSystem& h, int slot, const int seed[4], SlotMemory& mem, Staging& stg, long long vox_cap,
               int* vox_total, SysConst& Y, ChainDev& C, std::string& err, const SlotStart* start = nullptr);

class Batch {
 public:
  int device = 0;
  int tile = 0;  // kBatchTiles index of the launches
  cudaStream_t st = nullptr;
  std::vector<std::unique_ptr<Chain>> sys_chains;  // one opened chain per unique system
  std::vector<int> chain_sys;
  std::vector<SysConst> h_sys;
  SysConst* d_sys = nullptr;
  ChainDev* h_chains = nullptr;  // pinned host copy of every chain's control block
  ChainDev* d_chains = nullptr;
  std::vector<void*> allocations;
  MoveRecord* d_trace = nullptr;
  size_t trace_cap = 0;
  int kmax_all = 0, tab_sites = 0, tab_stride = 0, smem = 0;
  long long* d_timing = nullptr;  // per chain {start ns, end ns, SM} of the last launch
  long long* h_timing = nullptr;  // pinned host copy
  // placement of chains on CTAs: order[b] is the chain CTA b runs; after each launch it is
  // chosen again from that launch's SM map and per-chain times (rebalance)
  std::vector<int> order;
  int* d_order = nullptr;
  int* h_order = nullptr;         // pinned staging of order for the upload
  void rebalance();
  int nchains = 0;
  ~Batch();
  int open(const std::vector<std::string>& dirs, const std::vector<int>& seeds, int device, std::string& err,
           double voxel_edge = 2.0);
  // REVIVE + REVCON of chain c into outdir; restart of chain c from a REVIVE (call before
  // the chain's first run to match the reference's restart, which re-seeds duni).
  int write_revive(int c, const std::string& outdir, std::string& err);
  int restart(int c, const std::string& revive_path, std::string& err);
  // One step: control blocks host->device, `moves` moves of every chain, control blocks (and
  // the optional per-move trace) device->host.  *ms: CUDA-event time of the kernel alone.
  int run(int moves, MoveRecord* trace_host, float* ms, std::string& err);
  // numguests.out lines (gcmc.f:1937-1951) of chain c's last run, rebuilt from its move trace
  // and the per-species counts and energies the run started from
  int write_numguests(int c, const MoveRecord* trace, int nmoves, const std::string& outdir, bool append,
                      std::string& err) const;
  int profile = 0;
  std::vector<int> run_nmol;        // [chain][species] at the start of the last run
  std::vector<double> run_energy;   // [chain][species]
};

}  // namespace fmc
