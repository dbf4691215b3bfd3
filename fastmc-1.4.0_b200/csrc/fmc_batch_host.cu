// Host side of the batched path: deduplicated device systems, per-chain state, launches.
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>

#include "fmc_batch.h"
#include "fmc_restart.h"

namespace fmc {

namespace {

std::string slurp(const std::string& path) {
  std::ifstream f(path);
  std::stringstream ss;
  ss << f.rdbuf();
  return ss.str();
}

// Chains share a device system when framework, guests, force field, cell and the Ewald /
// cut-off parameters coincide; temperature, pressures and move mix stay per chain.
std::string system_key(const std::string& dir, const InputDeck& d) {
  std::ostringstream k;
  k.precision(17);
  k << slurp(dir + "/FIELD") << '\x1f' << slurp(dir + "/CONFIG") << '\x1f' << d.rcut << ' ' << d.rvdw << ' '
    << d.alpha << ' ' << d.delr << ' ' << d.kmax[0] << ' ' << d.kmax[1] << ' ' << d.kmax[2];
  return k.str();
}

}  // namespace

// Per-system constants from the host tables and the device arrays.
int fill_sysconst(const HostSystem& H, const DevSystem& S, SysConst& Y, int* tab_sites, std::string& err) {
  std::memset(&Y, 0, sizeof(Y));
  Y.S = S;
  Y.nspecies = (int)H.deck.guests.size();
  Y.ntypes = H.ntypes;
  Y.lrc_on = H.lrc_on;
  if (Y.ntypes > kBatchMaxTypes) {
    err = "more atom types than the batched path supports";
    return -5;
  }
  for (int g = 0; g < Y.nspecies; g++) {
    const GuestSpecies& G = H.deck.guests[g];
    if (G.nsite > kBatchMaxSites) {
      err = "guest with more sites than the batched path supports";
      return -5;
    }
    SpeciesConst& P = Y.sp[g];
    P.nsite = G.nsite;
    for (int s = 0; s < G.nsite; s++) {
      P.tx[s] = G.tx[s];
      P.ty[s] = G.ty[s];
      P.tz[s] = G.tz[s];
      P.q[s] = G.charge[s];
      P.mass[s] = G.mass[s];
      P.type[s] = G.type[s];
    }
    P.engsic = H.engsic[g];
    P.ewald3en = H.ewald3en[g];
    *tab_sites = std::max(*tab_sites, 2 * G.nsite);
  }
  for (int t = 1; t < (int)H.steadd.size() && t <= kBatchMaxTab; t++) Y.steadd[t] = H.steadd[t];
  for (int j = 0; j < H.nf; j++)
    if (H.ffrz[j]) Y.numfrz[H.ftype[j]]++;
  Y.engunit = H.engunit;
  Y.volm = H.cell.volm;
  Y.statvolm = H.statvolm;
  const InputDeck& d = H.deck;
  if ((int)d.plots.size() > kMaxPlots) {
    err = "more probability plots than the batched path supports";
    return -5;
  }
  Y.nplots = (int)d.plots.size();
  for (int a = 0; a < 3; a++) Y.ngrid[a] = d.ngrid[a];
  for (int ip = 0; ip < Y.nplots; ip++) {
    if ((int)d.plots[ip].sites.size() > kMaxPlotSites) {
      err = "a probability plot lists more sites than the batched path supports";
      return -5;
    }
    Y.plot_guest[ip] = d.plots[ip].guest;
    Y.plot_nsite[ip] = (int)d.plots[ip].sites.size();
    for (size_t j = 0; j < d.plots[ip].sites.size(); j++) Y.plot_site[ip][j] = d.plots[ip].sites[j];
  }
  return 0;
}

// Per-system constants of an opened system chain (its HostSystem and device arrays).
int make_sysconst(const Chain& ch, SysConst& Y, std::vector<void*>& allocations, int* tab_sites, std::string& err) {
  (void)allocations;
  return fill_sysconst(ch.sys, ch.dsys.view, Y, tab_sites, err);
}

// Parameters (from the chain's own deck) and initial state of one chain of system `sys`;
// allocates its S(k) (a copy of sk_src, the framework's) and guest-site segments.
size_t chain_state_bytes(const InputDeck& d, const HostSystem& H, bool record_samples) {
  const size_t ng = d.guests.size(), sites = std::max<size_t>(ng * (size_t)d.maxguest, 1);
  size_t b = sizeof(double2) * std::max(H.K, 1) + (sizeof(double4) + sizeof(int)) * sites;
  if (record_samples) b += 2 * sizeof(double) * (ng * (size_t)kSampleCap + 1);
  if (!H.deck.plots.empty())
    b += sizeof(unsigned long long) * H.deck.plots.size() * (size_t)H.deck.ngrid[0] * H.deck.ngrid[1] *
         H.deck.ngrid[2];
  return b;
}

int init_chain_state(const InputDeck& d, const HostSystem& H, const double2* sk_src, double energy0, int sys,
                     const int* seed, ChainDev& C, const DevAllocFn& alloc, cudaStream_t st, std::string& err,
                     bool record_samples) {
  std::memset(&C, 0, sizeof(C));
  C.sys = sys;
  C.temp = d.temp;
  C.beta = 1.0 / (kKboltz * d.temp);
  const int ng = (int)d.guests.size();
  for (int g = 0; g < ng; g++) {
    C.press[g] = d.press[g];
    std::array<double, 9> f = d.movefreq[g];
    double nrm = 0;
    for (double v : f) nrm += v;
    if (nrm == 0) {
      nrm = 1;
      f = {1.0 / 3.0, 1.0 / 3.0, 1.0 / 3.0, 0, 0, 0, 0, 0, 0};
    }
    C.mvcum[g][0] = f[0] / nrm;
    for (int k = 1; k < 9; k++) C.mvcum[g][k] = C.mvcum[g][k - 1] + (f[k] / nrm);
    C.disp_ratio[g] = d.disp_ratio[g];
    C.tran_ratio[g] = d.tran_ratio[g];
    C.delrdisp[g] = d.delr;
    C.tran_delr[g] = d.delr;
    C.energy[g] = energy0;
  }
  C.rota_ratio = d.rota_ratio;
  C.despre = d.despre;
  C.packf = d.packf;
  for (int g = 0; g < ng; g++) {
    C.adspres[g] = d.adspres[g];
    C.adsguen[g] = d.adsguen[g];
  }
  C.maxguest = d.maxguest;
  C.mcsteps = d.mcsteps;
  C.eqsteps = d.eqsteps;
  C.nwind = d.nwind;
  C.laccsample = d.laccsample;
  duni_seed(C.rng, seed[0], seed[1], seed[2], seed[3]);
  duni_next(C.rng);  // gcmc.f:335-336
  C.totatm = C.framatm = H.nf;
  for (int j = 0; j < H.nf; j++) C.numtyp[H.ftype[j]]++;
  C.rotangle = kPi / 3.0;
  C.rota_rotangle = kPi / 3.0;
  C.production = d.eqsteps == 0;
  C.lgchk = 1;
  C.active = 1;
  C.budget = 0;
  // buffers: S(k) starts as the system's (framework plus any guests the deck preloads), guest
  // segments per species
  cudaError_t e = alloc((void**)&C.sk, sizeof(double2) * std::max(H.K, 1));
  if (e == cudaSuccess) e = cudaMemcpyAsync(C.sk, sk_src, sizeof(double2) * H.K, cudaMemcpyDeviceToDevice, st);
  int off = 0;
  for (int g = 0; g < ng; g++) {
    C.seg_off[g] = off;
    C.seg_cap[g] = d.maxguest;
    off += d.maxguest;
  }
  if (e == cudaSuccess) e = alloc((void**)&C.gsite, sizeof(double4) * std::max(off, 1));
  if (e == cudaSuccess) e = alloc((void**)&C.gtype, sizeof(int) * std::max(off, 1));
  if (e == cudaSuccess && record_samples) {  // gasmol / gaseng of the final report
    const size_t n = (size_t)ng * kSampleCap + 1;
    e = alloc((void**)&C.gasmol, sizeof(double) * n);
    if (e == cudaSuccess) e = alloc((void**)&C.gaseng, sizeof(double) * n);
    if (e == cudaSuccess) e = cudaMemsetAsync(C.gasmol, 0, sizeof(double) * n, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(C.gaseng, 0, sizeof(double) * n, st);
  }
  if (e == cudaSuccess && !H.deck.plots.empty()) {
    const size_t n = H.deck.plots.size() * (size_t)H.deck.ngrid[0] * H.deck.ngrid[1] * H.deck.ngrid[2];
    e = alloc((void**)&C.prob, sizeof(unsigned long long) * n);
    if (e == cudaSuccess) e = cudaMemsetAsync(C.prob, 0, sizeof(unsigned long long) * n, st);
  }
  if (e != cudaSuccess) {
    err = std::string("batch allocation failed: ") + cudaGetErrorString(e);
    return -100 - (int)e;
  }
  return 0;
}

int init_chain(const InputDeck& d, const Chain& ch, int sys, const int* seed, ChainDev& C,
               std::vector<void*>& allocations, cudaStream_t st, std::string& err) {
  DevAllocFn alloc = [&allocations](void** p, size_t n) {
    cudaError_t e = cudaMalloc(p, n);
    if (e == cudaSuccess) allocations.push_back(*p);
    return e;
  };
  int rc = init_chain_state(d, ch.sys, ch.sk, ch.spenergy, sys, seed, C, alloc, st, err, true);
  if (rc) return rc;
  // guests preloaded by the deck (FIELD NUMMOLS > 0 with their sites in CONFIG): the system's
  // chain already holds them in S(k) and in the single-point energy; copy their sites
  for (size_t g = 0; g < ch.sp.size(); g++) {
    const GuestSpecies& G = ch.sys.deck.guests[g];
    const int n = ch.sp[g].nmol * G.nsite;
    if (n == 0) continue;
    if (n > C.seg_cap[g]) {
      err = "preloaded guests exceed the chain's capacity (max guest atoms)";
      return -75;
    }
    std::vector<double4> a(n);
    std::vector<int> t(n);
    for (int i = 0; i < n; i++) {
      a[i] = make_double4(ch.sp[g].xyz[3 * i], ch.sp[g].xyz[3 * i + 1], ch.sp[g].xyz[3 * i + 2],
                          G.charge[i % G.nsite]);
      t[i] = G.type[i % G.nsite];
      C.numtyp[t[i]]++;
    }
    cudaError_t e = cudaMemcpy(C.gsite + C.seg_off[g], a.data(), sizeof(double4) * n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(C.gtype + C.seg_off[g], t.data(), sizeof(int) * n, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
      err = std::string("preloaded guest upload failed: ") + cudaGetErrorString(e);
      return -100 - (int)e;
    }
    C.nmol[g] = ch.sp[g].nmol;
    C.totatm += n;
  }
  return 0;
}

Batch::~Batch() {
  if (st) {
    cudaSetDevice(device);
    cudaStreamSynchronize(st);
    for (void* p : allocations) cudaFree(p);
    if (d_trace) cudaFree(d_trace);
    if (h_chains) cudaFreeHost(h_chains);
    if (h_timing) cudaFreeHost(h_timing);
    if (h_order) cudaFreeHost(h_order);
    cudaStreamDestroy(st);
  }
}

int Batch::open(const std::vector<std::string>& dirs, const std::vector<int>& seeds, int dev, std::string& err,
                double voxel_edge) {
  device = dev;
  nchains = (int)dirs.size();
  if (cudaSetDevice(dev) != cudaSuccess || cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) {
    err = "cannot select the device";
    return -100;
  }
  std::map<std::string, int> sys_of_key;
  std::vector<InputDeck> decks(nchains);
  chain_sys.assign(nchains, 0);
  for (int c = 0; c < nchains; c++) {
    int rc = read_input_deck(dirs[c], decks[c], err);
    if (rc) {
      err = dirs[c] + ": " + err;
      return rc;
    }
    std::string key = system_key(dirs[c], decks[c]);
    auto it = sys_of_key.find(key);
    if (it == sys_of_key.end()) {
      auto ch = std::make_unique<Chain>();
      int s4[4] = {12, 34, 56, 78};
      rc = ch->open(dirs[c], s4, dev, err, voxel_edge);
      if (rc) {
        err = dirs[c] + ": " + err;
        return rc;
      }
      int id = (int)sys_chains.size();
      sys_chains.push_back(std::move(ch));
      sys_of_key[key] = id;
      chain_sys[c] = id;
    } else {
      chain_sys[c] = it->second;
    }
  }
  // ---- per-system constants
  h_sys.assign(sys_chains.size(), SysConst());
  for (size_t i = 0; i < sys_chains.size(); i++) {
    int rc = make_sysconst(*sys_chains[i], h_sys[i], allocations, &tab_sites, err);
    if (rc) return rc;
    const HostSystem& H = sys_chains[i]->sys;
    kmax_all = std::max(kmax_all, H.K);
    tab_stride = std::max(tab_stride, H.deck.kmax[0] + H.deck.kmax[1] + H.deck.kmax[2] + 3);
  }
  kmax_all = (kmax_all + 3) & ~3;
  smem = batch_smem_bytes(kmax_all, tab_sites, tab_stride);
  if (smem > 220 * 1024) {
    err = "k-vector tables of this batch exceed the shared-memory budget of one CTA";
    return -9;
  }
  if (configure_batch_kernel(smem) != cudaSuccess) {
    err = "cannot configure the batched kernel";
    return -100;
  }
  // ---- per-chain state
  if (cudaMallocHost(&h_chains, sizeof(ChainDev) * nchains) != cudaSuccess) {
    err = "cannot allocate pinned host memory for the chain control blocks";
    return -100;
  }
  for (int c = 0; c < nchains; c++) {
    int rc = init_chain(decks[c], *sys_chains[chain_sys[c]], chain_sys[c], &seeds[4 * c], h_chains[c], allocations,
                        st, err);
    if (rc) return rc;
  }
  cudaError_t e = cudaMalloc(&d_sys, sizeof(SysConst) * h_sys.size());
  if (e == cudaSuccess) allocations.push_back(d_sys);
  if (e == cudaSuccess) e = cudaMemcpy(d_sys, h_sys.data(), sizeof(SysConst) * h_sys.size(), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMalloc(&d_chains, sizeof(ChainDev) * nchains);
  if (e == cudaSuccess) allocations.push_back(d_chains);
  if (e == cudaSuccess) e = cudaMemcpy(d_chains, h_chains, sizeof(ChainDev) * nchains, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMalloc(&d_timing, sizeof(long long) * 3 * nchains);
  if (e == cudaSuccess) allocations.push_back(d_timing);
  if (e == cudaSuccess) e = cudaMemset(d_timing, 0, sizeof(long long) * 3 * nchains);
  if (e == cudaSuccess) e = cudaMallocHost(&h_timing, sizeof(long long) * 3 * nchains);
  if (e == cudaSuccess) std::memset(h_timing, 0, sizeof(long long) * 3 * nchains);
  if (e == cudaSuccess) e = cudaMalloc(&d_order, sizeof(int) * nchains);
  if (e == cudaSuccess) allocations.push_back(d_order);
  if (e == cudaSuccess) e = cudaMallocHost(&h_order, sizeof(int) * nchains);
  order.resize(nchains);
  for (int c = 0; c < nchains; c++) order[c] = c;
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    err = std::string("batch upload failed: ") + cudaGetErrorString(e);
    return -100 - (int)e;
  }
  return 0;
}

int Batch::write_revive(int c, const std::string& outdir, std::string& err) {
  const ChainDev& C = h_chains[c];
  const Chain& S = *sys_chains[chain_sys[c]];
  const InputDeck& d = S.sys.deck;
  const int ng = (int)d.guests.size();
  std::vector<std::vector<double>> xyz(ng);
  cudaSetDevice(device);
  for (int g = 0; g < ng; g++) {
    const int n = C.nmol[g] * d.guests[g].nsite;
    std::vector<double4> a(std::max(n, 1));
    if (n) {
      cudaError_t e = cudaMemcpy(a.data(), C.gsite + C.seg_off[g], sizeof(double4) * n, cudaMemcpyDeviceToHost);
      if (e != cudaSuccess) {
        err = cudaGetErrorString(e);
        return -100 - (int)e;
      }
    }
    for (int i = 0; i < n; i++) {
      xyz[g].push_back(a[i].x);
      xyz[g].push_back(a[i].y);
      xyz[g].push_back(a[i].z);
    }
  }
  std::vector<double> cs(1 + 14 * ng, 0.0), en(ng);
  cs[0] = (double)C.prodcount;
  for (int g = 0; g < ng; g++) {
    for (int k = 0; k < 6; k++) cs[1 + 14 * g + k] = C.stats[g][k];
    en[g] = C.energy[g];
  }
  Revive r = revive_state(d, C.production != 0, xyz, cs, en);
  int rc = fmc::write_revive(outdir + "/REVIVE", r, err);
  if (!rc) rc = fmc::write_revcon(outdir + "/REVCON", d, r, C.last_dE, err);
  return rc;
}

int Batch::restart(int c, const std::string& path, std::string& err) {
  ChainDev& C = h_chains[c];
  Chain& S = *sys_chains[chain_sys[c]];
  const InputDeck& d = S.sys.deck;
  const int ng = (int)d.guests.size();
  Revive r;
  int rc = read_revive(path, d, r, err);
  if (rc) return rc;
  const std::vector<std::vector<double>> xyz = revive_guest_xyz(d, r);
  for (int g = 0; g < ng; g++)
    if ((int)(xyz[g].size() / 3) > C.seg_cap[g]) {
      err = "REVIVE holds more guests than the chain's capacity (max guest atoms)";
      return -75;
    }
  // the system's own chain computes the single point and S(k) of the restart state
  cudaSetDevice(device);
  rc = S.restart(r, err);
  if (rc) return rc;
  cudaError_t e = cudaMemcpy(C.sk, S.sk, sizeof(double2) * S.sys.K, cudaMemcpyDeviceToDevice);
  for (int g = 0; g < ng && e == cudaSuccess; g++) {
    const GuestSpecies& G = d.guests[g];
    const int n = (int)(xyz[g].size() / 3);
    std::vector<double4> a(std::max(n, 1));
    std::vector<int> t(std::max(n, 1));
    for (int i = 0; i < n; i++) {
      a[i] = make_double4(xyz[g][3 * i], xyz[g][3 * i + 1], xyz[g][3 * i + 2], G.charge[i % G.nsite]);
      t[i] = G.type[i % G.nsite];
    }
    if (n) e = cudaMemcpy(C.gsite + C.seg_off[g], a.data(), sizeof(double4) * n, cudaMemcpyHostToDevice);
    if (n && e == cudaSuccess) e = cudaMemcpy(C.gtype + C.seg_off[g], t.data(), sizeof(int) * n, cudaMemcpyHostToDevice);
  }
  if (e != cudaSuccess) {
    err = std::string("restart upload failed: ") + cudaGetErrorString(e);
    return -100 - (int)e;
  }
  const HostSystem& H = S.sys;
  std::memset(C.numtyp, 0, sizeof(C.numtyp));
  for (int j = 0; j < H.nf; j++) C.numtyp[H.ftype[j]]++;
  C.totatm = H.nf;
  for (int g = 0; g < ng; g++) {
    const GuestSpecies& G = d.guests[g];
    C.nmol[g] = (int)(xyz[g].size() / (3 * G.nsite));
    C.totatm += C.nmol[g] * G.nsite;
    for (int m = 0; m < C.nmol[g]; m++)
      for (int i = 0; i < G.nsite; i++) C.numtyp[G.type[i]]++;
    C.energy[g] = S.spenergy;  // gcmc.f:547-556
    for (int k = 0; k < 6; k++) C.stats[g][k] = r.chainstats[1 + 14 * g + k];
  }
  C.framatm = H.nf;
  C.prodcount = 0;
  C.last_dE = 0.0;
  C.production = r.production;
  if (C.production && C.eqsteps > 0) C.production = 0;  // gcmc.f:396-409
  if (C.eqsteps == 0) C.production = 1;                 // gcmc.f:553-554
  // the system chain is left without guests: the batch's chains no longer read its state
  for (int g = 0; g < ng; g++) S.set_guests(g, 0, nullptr);
  return 0;
}

int Batch::write_numguests(int c, const MoveRecord* trace, int nmoves, const std::string& outdir, bool append,
                           std::string& err) const {
  const InputDeck& d = sys_chains[chain_sys[c]]->sys.deck;
  const int ng = (int)d.guests.size();
  if ((int)run_nmol.size() < kMaxGuestTypes * nchains) {
    err = "the batch has not run yet";
    return -1;
  }
  int nmol[kMaxGuestTypes];
  double eng[kMaxGuestTypes];
  for (int i = 0; i < ng; i++) {
    nmol[i] = run_nmol[(size_t)c * kMaxGuestTypes + i];
    eng[i] = run_energy[(size_t)c * kMaxGuestTypes + i];
  }
  std::vector<std::FILE*> f(ng, nullptr);
  for (int i = 0; i < ng; i++) {
    char a[64];
    if (ng > 1) std::snprintf(a, sizeof(a), "/numguests%02d.out", i + 1);
    else std::snprintf(a, sizeof(a), "/numguests.out");
    f[i] = std::fopen((outdir + a).c_str(), append ? "a" : "w");
    if (!f[i]) {
      err = "cannot write numguests.out under " + outdir;
      for (std::FILE* h : f)
        if (h) std::fclose(h);
      return -1;
    }
  }
  for (int m = 0; m < nmoves; m++) {
    const MoveRecord& r = trace[m];
    if (r.mtype == 0) break;  // the chain finished before this record
    const int g = r.iguest;
    nmol[g] = r.nmols_after;
    eng[g] = r.energy_after;
    if (r.step % d.nnumg != 0) continue;
    int fl[6] = {0, 0, 0, 0, 0, 0};
    if (r.mtype == kInsert) fl[0] = 1;
    else if (r.mtype == kDelete) fl[1] = 1;
    else if (r.mtype == kDisplace) fl[2] = 1;
    else if (r.mtype == kTranslate) fl[2] = 2;
    else if (r.mtype == kRotate) fl[2] = 3;
    else if (r.mtype == kJump) fl[3] = 1;
    else if (r.mtype == kMultiJump) fl[3] = 2;
    const double de = (r.mtype != kNoop && r.accepted) ? r.estep : 0.0;
    for (int i = 0; i < ng; i++) {
      const bool me = i == g;
      std::fprintf(f[i], "%9d%7d%20.6f%20.6f%4d%4d%4d%4d%4d%4d\n", r.step, nmol[i], eng[i], me ? de : 0.0,
                   me ? fl[0] : 0, me ? fl[1] : 0, me ? fl[2] : 0, me ? fl[3] : 0, me ? fl[4] : 0, me ? fl[5] : 0);
    }
  }
  for (std::FILE* h : f) std::fclose(h);
  return 0;
}

// Placement for the next launch from the one that just ran.  The GPU places CTAs on SMs in block
// order, the same way launch after launch: with more chains than SMs, some SMs run two CTAs, each
// of them then slower (about 12%), and the launch lasts as long as its slowest CTA.  So the
// heaviest chains (per-chain device time of the last launch, with the sharing factor taken out)
// go to the blocks that had an SM of their own, and the remaining blocks, two per SM, pair the
// heaviest remaining chain with the lightest.  With a different placement the assignment is only
// less balanced; every chain computes the same moves wherever it runs.
void Batch::rebalance() {
  const int n = nchains;
  std::map<long long, std::vector<int>> by_sm;  // SM -> blocks
  for (int b = 0; b < n; b++) {
    const long long* t = h_timing + 3 * order[b];
    if (t[1] <= t[0]) return;  // a CTA without a record: keep the placement
    by_sm[t[2]].push_back(b);
  }
  std::vector<double> cost(n);
  for (auto& kv : by_sm) {
    if (kv.second.size() > 2) return;  // more CTAs on an SM than fit at once: placement not learned
    for (int b : kv.second) {
      const long long* t = h_timing + 3 * order[b];
      cost[order[b]] = (double)(t[1] - t[0]) / (kv.second.size() == 2 ? 1.12 : 1.0);
    }
  }
  std::vector<int> chains(n);
  for (int c = 0; c < n; c++) chains[c] = c;
  std::stable_sort(chains.begin(), chains.end(), [&cost](int x, int y) { return cost[x] > cost[y]; });
  std::vector<int> single, paired_a, paired_b;
  for (auto& kv : by_sm) {
    if (kv.second.size() == 1) {
      single.push_back(kv.second[0]);
    } else {
      paired_a.push_back(kv.second[0]);
      paired_b.push_back(kv.second[1]);
    }
  }
  std::sort(single.begin(), single.end());
  std::vector<int> next(n);
  size_t k = 0;
  for (int b : single) next[b] = chains[k++];
  const size_t np = paired_a.size();
  for (size_t i = 0; i < np; i++) {
    next[paired_a[i]] = chains[k + i];
    next[paired_b[i]] = chains[n - 1 - i];
  }
  order = next;
}

int Batch::run(int moves, MoveRecord* trace_host, float* ms, std::string& err) {
  cudaSetDevice(device);
  run_nmol.resize((size_t)kMaxGuestTypes * nchains);
  run_energy.resize((size_t)kMaxGuestTypes * nchains);
  for (int c = 0; c < nchains; c++)
    for (int i = 0; i < kMaxGuestTypes; i++) {
      run_nmol[(size_t)c * kMaxGuestTypes + i] = h_chains[c].nmol[i];
      run_energy[(size_t)c * kMaxGuestTypes + i] = h_chains[c].energy[i];
    }
  BatchLaunch L;
  std::memset(&L, 0, sizeof(L));
  L.chains = d_chains;
  L.systems = d_sys;
  L.nchains = nchains;
  L.moves = moves;
  L.kmax_smem = kmax_all;
  L.profile = profile;
  L.trace = nullptr;
  L.timing = d_timing;
  L.order = d_order;
  L.tile = tile;
  cudaError_t e = cudaSuccess;
  if (trace_host) {
    size_t need = (size_t)nchains * moves;
    if (need > trace_cap) {
      if (d_trace) cudaFree(d_trace);
      d_trace = nullptr;
      e = cudaMalloc(&d_trace, sizeof(MoveRecord) * need);
      trace_cap = e == cudaSuccess ? need : 0;
    }
    L.trace = d_trace;
  }
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  const size_t cb = sizeof(ChainDev) * nchains;
  std::copy(order.begin(), order.end(), h_order);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_order, h_order, sizeof(int) * nchains, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_chains, h_chains, cb, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaEventRecord(a, st);
  if (e == cudaSuccess) e = launch_batch(L, smem, tab_stride, st);
  if (e == cudaSuccess) e = cudaEventRecord(b, st);
  if (e == cudaSuccess && trace_host)
    e = cudaMemcpyAsync(trace_host, d_trace, sizeof(MoveRecord) * (size_t)nchains * moves, cudaMemcpyDeviceToHost,
                        st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(h_chains, d_chains, cb, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(h_timing, d_timing, sizeof(long long) * 3 * nchains, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  float t = 0.f;
  if (e == cudaSuccess) cudaEventElapsedTime(&t, a, b);
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  if (e != cudaSuccess) {
    err = std::string("batched launch failed: ") + cudaGetErrorString(e);
    return -100 - (int)e;
  }
  rebalance();
  if (ms) *ms = t;
  return 0;
}

}  // namespace fmc

// ============================================================== C ABI of the batched path
#include "../../include/fastmc_b200.h"

namespace fmc {
void set_last_error(const std::string& msg);
}

struct fmc_batch {
  fmc::Batch impl;
};

namespace {

// CONTROL `restart` on a batch: the chains opened from one deck directory are that job's
// nodes, numbered in the order they appear; each reads its branch REVIVE (gcmc.f:353-394)
// before its first run, as fmc_batch_restart does.
int restart_from_branches(fmc::Batch& B, const std::vector<std::string>& dirs, std::string& err) {
  std::map<std::string, int> seen;
  for (int c = 0; c < B.nchains; c++) {
    const int node = seen[dirs[c]]++;
    const fmc::InputDeck& d = B.sys_chains[B.chain_sys[c]]->sys.deck;
    if (!d.lrestart || d.lspe) continue;
    fmc::BranchChoice ch;
    int rc = fmc::choose_branch(dirs[c], node, ch, err);
    if (!rc && !ch.revive.empty()) rc = B.restart(c, ch.revive, err);
    if (rc) {
      err = dirs[c] + ": " + err;
      return rc;
    }
  }
  return 0;
}

}  // namespace

extern "C" {

int fmc_batch_control_block_bytes(void) { return (int)sizeof(fmc::ChainDev); }
int fmc_system_block_bytes(void) { return (int)sizeof(fmc::SysConst); }

int fmc_batch_open(int nchains, const char* const* dirs, const int* seeds, int device, fmc_batch** out) {
  if (!dirs || !seeds || !out || nchains < 1) {
    fmc::set_last_error("null argument or empty batch");
    return -1;
  }
  fmc_batch* b = new fmc_batch();
  std::vector<std::string> d(dirs, dirs + nchains);
  std::vector<int> s(seeds, seeds + 4 * nchains);
  std::string err;
  int rc = b->impl.open(d, s, device, err);
  if (!rc) rc = restart_from_branches(b->impl, d, err);
  if (rc) {
    delete b;
    *out = nullptr;
    fmc::set_last_error(err);
    return rc;
  }
  *out = b;
  return 0;
}

int fmc_batch_open_edge(int nchains, const char* const* dirs, const int* seeds, int device, double voxel_edge,
                        fmc_batch** out) {
  if (!dirs || !seeds || !out || nchains < 1 || !(voxel_edge >= 0.5 && voxel_edge <= 8.0)) {
    fmc::set_last_error("null argument, empty batch or voxel edge outside 0.5-8 A");
    return -1;
  }
  fmc_batch* b = new fmc_batch();
  std::vector<std::string> d(dirs, dirs + nchains);
  std::vector<int> s(seeds, seeds + 4 * nchains);
  std::string err;
  int rc = b->impl.open(d, s, device, err, voxel_edge);
  if (!rc) rc = restart_from_branches(b->impl, d, err);
  if (rc) {
    delete b;
    *out = nullptr;
    fmc::set_last_error(err);
    return rc;
  }
  *out = b;
  return 0;
}

int fmc_batch_autotune(int nchains, const char* const* dirs, const int* seeds, int device, const double* edges,
                       int nedges, int moves, double* best_edge, float* ms) {
  if (!dirs || !seeds || !edges || nedges < 1 || moves < 1 || !best_edge) {
    fmc::set_last_error("bad autotune arguments");
    return -1;
  }
  // every candidate on a throwaway batch of the same chains: one warm-up launch, one timed
  double best = 0.0;
  float best_ms = 0.0f;
  for (int i = 0; i < nedges; i++) {
    fmc_batch* b = nullptr;
    int rc = fmc_batch_open_edge(nchains, dirs, seeds, device, edges[i], &b);
    float t = 0.0f;
    if (!rc) rc = fmc_batch_run(b, moves, nullptr, &t);
    if (!rc) rc = fmc_batch_run(b, moves, nullptr, &t);
    if (b) fmc_batch_close(b);
    if (rc) return rc;
    if (ms) ms[i] = t;
    if (i == 0 || t < best_ms) {
      best = edges[i];
      best_ms = t;
    }
  }
  *best_edge = best;
  return 0;
}

void fmc_batch_close(fmc_batch* b) { delete b; }

int fmc_batch_profile(fmc_batch* b, int enable) {
  if (!b) {
    fmc::set_last_error("bad batch handle");
    return -1;
  }
  if (enable && b->impl.tile != 0) {
    fmc::set_last_error("phase profiling is built for the default tile (0) only");
    return -1;
  }
  b->impl.profile = enable;
  return 0;
}

int fmc_batch_tiles(int* threads, int* kvec_per_trip, int* cand_per_trip, int cap) {
  for (int t = 0; t < fmc::kNumBatchTiles && t < cap; t++) {
    if (threads) threads[t] = fmc::kBatchTiles[t].threads;
    if (kvec_per_trip) kvec_per_trip[t] = fmc::kBatchTiles[t].kvec_per_trip;
    if (cand_per_trip) cand_per_trip[t] = fmc::kBatchTiles[t].cand_per_trip;
  }
  return fmc::kNumBatchTiles;
}

int fmc_batch_set_tile(fmc_batch* b, int tile) {
  if (!b || tile < 0 || tile >= fmc::kNumBatchTiles) {
    fmc::set_last_error("bad batch handle or tile index");
    return -1;
  }
  if (tile != 0 && b->impl.profile) {
    fmc::set_last_error("phase profiling is built for the default tile (0) only");
    return -1;
  }
  b->impl.tile = tile;
  return 0;
}

int fmc_batch_get_tile(fmc_batch* b) { return b ? b->impl.tile : -1; }

int fmc_batch_autotune_tiles(int nchains, const char* const* dirs, const int* seeds, int device, double voxel_edge,
                             const int* tiles, int ntiles, int warm_moves, int moves, int* best_tile, float* ms) {
  if (!dirs || !seeds || !tiles || ntiles < 1 || moves < 1 || warm_moves < 0 || !best_tile) {
    fmc::set_last_error("bad autotune arguments");
    return -1;
  }
  for (int i = 0; i < ntiles; i++)
    if (tiles[i] < 0 || tiles[i] >= fmc::kNumBatchTiles) {
      fmc::set_last_error("tile index out of range");
      return -1;
    }
  // one throwaway batch of the same chains: warmed up, then every tile launched twice in
  // palindromic order (t0 .. tn-1, tn-1 .. t0) so that the chains' drift over the runs (they
  // fill with guests) weighs on every tile alike; a tile's time is the mean of its two launches
  fmc_batch* b = nullptr;
  int rc = fmc_batch_open_edge(nchains, dirs, seeds, device, voxel_edge, &b);
  float t = 0.0f;
  if (!rc && warm_moves > 0) rc = fmc_batch_run(b, warm_moves, nullptr, &t);
  std::vector<float> sum(ntiles, 0.0f);
  for (int pass = 0; pass < 2 && !rc; pass++)
    for (int j = 0; j < ntiles && !rc; j++) {
      const int i = pass == 0 ? j : ntiles - 1 - j;
      rc = fmc_batch_set_tile(b, tiles[i]);
      if (!rc) rc = fmc_batch_run(b, moves, nullptr, &t);
      sum[i] += t;
    }
  if (b) fmc_batch_close(b);
  if (rc) return rc;
  int best = 0;
  for (int i = 0; i < ntiles; i++) {
    if (ms) ms[i] = 0.5f * sum[i];
    if (sum[i] < sum[best]) best = i;
  }
  *best_tile = tiles[best];
  return 0;
}

int fmc_batch_run(fmc_batch* b, int moves, fmc_move_record* trace, float* device_ms) {
  if (!b || moves < 0) {
    fmc::set_last_error("bad batch handle or move count");
    return -1;
  }
  std::string err;
  int rc = b->impl.run(moves, reinterpret_cast<fmc::MoveRecord*>(trace), device_ms, err);
  if (rc) {
    fmc::set_last_error(err);
    return rc;
  }
  for (int i = 0; i < b->impl.nchains; i++) {
    const fmc::ChainDev& c = b->impl.h_chains[i];
    if (c.status) {
      fmc::set_last_error(c.status == 75 ? "too many atoms in specified system" : "chain stopped with an unknown status");
      return c.status;
    }
  }
  return 0;
}

int fmc_batch_chain_state(fmc_batch* b, int chain, double* out) {
  if (!b || chain < 0 || chain >= b->impl.nchains || !out) {
    fmc::set_last_error("bad batch handle or chain index");
    return -1;
  }
  const fmc::ChainDev& C = b->impl.h_chains[chain];
  double v[40] = {0};
  v[0] = C.status;
  v[1] = (double)C.moves_done;
  v[2] = C.gcmccount;
  for (int g = 0; g < fmc::kMaxGuestTypes; g++) {
    v[3 + g] = C.nmol[g];
    v[7 + g] = C.energy[g];
  }
  v[11] = C.elrc;
  v[12] = C.accept_ins;
  v[13] = C.accept_del;
  v[14] = C.ins_count;
  v[15] = C.del_count;
  v[16] = (double)C.prodcount;
  for (int k = 0; k < 5; k++) v[17 + k] = C.stats[0][k];
  v[22] = C.sys;
  v[23] = b->impl.h_sys[C.sys].S.K;
  v[24] = b->impl.h_sys[C.sys].S.nf;
  v[25] = C.temp;
  v[26] = C.press[0];
  for (int k = 0; k < 5; k++) v[27 + k] = (double)C.prof[k];
  for (int k = 5; k < 9; k++) v[k + 27] = (double)C.prof[k];
  v[36] = C.lgchk ? 0.0 : 1.0;
  std::memcpy(out, v, sizeof(v));
  return 0;
}

int fmc_batch_chain_timing(fmc_batch* b, int chain, long long* out) {
  if (!b || chain < 0 || chain >= b->impl.nchains || !out) {
    fmc::set_last_error("bad batch handle or chain index");
    return -1;
  }
  for (int k = 0; k < 3; k++) out[k] = b->impl.h_timing ? b->impl.h_timing[3 * chain + k] : 0;
  return 0;
}

int fmc_batch_voxels(fmc_batch* b, int chain, int* nvox, int* off, int* atoms, long long cap, long long* n_entries) {
  if (!b || chain < 0 || chain >= b->impl.nchains || !nvox || !n_entries) {
    fmc::set_last_error("bad batch handle, chain index or argument");
    return -1;
  }
  const fmc::Chain& sc = *b->impl.sys_chains[b->impl.chain_sys[chain]];
  const fmc::DevSystem& v = sc.dsys.view;
  for (int a = 0; a < 3; a++) nvox[a] = v.nvox[a];
  *n_entries = sc.dsys.vox_entries;
  const int nv = v.nvox[0] * v.nvox[1] * v.nvox[2];
  cudaSetDevice(b->impl.device);
  cudaError_t e = cudaSuccess;
  if (off) e = cudaMemcpy(off, v.vox_off, sizeof(int) * (nv + 1), cudaMemcpyDeviceToHost);
  if (atoms && e == cudaSuccess) {
    if (cap < sc.dsys.vox_entries) {
      fmc::set_last_error("atoms buffer smaller than the voxel entries");
      return -2;
    }
    if (sc.dsys.vox_entries)
      e = cudaMemcpy(atoms, v.vox_atoms, sizeof(int) * sc.dsys.vox_entries, cudaMemcpyDeviceToHost);
  }
  if (e != cudaSuccess) {
    fmc::set_last_error(cudaGetErrorString(e));
    return -100 - (int)e;
  }
  return 0;
}

int fmc_batch_prob(fmc_batch* b, int chain, int plot, int* dims, double* out) {
  if (!b || chain < 0 || chain >= b->impl.nchains) {
    fmc::set_last_error("bad batch handle or chain index");
    return -1;
  }
  const fmc::Batch& B = b->impl;
  const fmc::ChainDev& C = B.h_chains[chain];
  const fmc::InputDeck& d = B.sys_chains[B.chain_sys[chain]]->sys.deck;
  const size_t cells = (size_t)d.ngrid[0] * d.ngrid[1] * d.ngrid[2];
  if (dims) {
    dims[0] = (int)d.plots.size();
    for (int a = 0; a < 3; a++) dims[1 + a] = d.ngrid[a];
  }
  if (out) {
    if (plot < 0 || plot >= (int)d.plots.size()) {
      fmc::set_last_error("plot index out of range");
      return -1;
    }
    std::vector<unsigned long long> q(cells);
    cudaSetDevice(B.device);
    cudaError_t e = cudaMemcpy(q.data(), C.prob + plot * cells, sizeof(unsigned long long) * cells,
                               cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) {
      fmc::set_last_error(cudaGetErrorString(e));
      return -100 - (int)e;
    }
    for (size_t i = 0; i < cells; i++) out[i] = (double)q[i] / 4294967296.0;
  }
  return 0;
}

int fmc_batch_write_prob(fmc_batch* b, int chain, const char* outdir) {
  if (!b || chain < 0 || chain >= b->impl.nchains || !outdir) {
    fmc::set_last_error("bad batch handle, chain index or directory");
    return -1;
  }
  const fmc::Batch& B = b->impl;
  const fmc::ChainDev& C = B.h_chains[chain];
  const fmc::InputDeck& d = B.sys_chains[B.chain_sys[chain]]->sys.deck;
  if (C.prodcount <= 0) return 0;
  const size_t cells = (size_t)d.ngrid[0] * d.ngrid[1] * d.ngrid[2];
  std::vector<double> grid(cells);
  std::vector<int> per(d.guests.size(), 0);
  for (size_t ip = 0; ip < d.plots.size(); ip++) {
    int rc = fmc_batch_prob(b, chain, (int)ip, nullptr, grid.data());
    if (rc) return rc;
    const int g = d.plots[ip].guest;
    char name[64];
    std::snprintf(name, sizeof(name), "/prob_guest%02d_prob_%02d.cube", g + 1, ++per[g]);
    std::string err;
    rc = fmc::write_prob_cube(std::string(outdir) + name, d, grid.data(), C.prodcount, err);
    if (rc) {
      fmc::set_last_error(err);
      return rc;
    }
  }
  return 0;
}

namespace {
// The chainstats layout of a batched chain, with its stored samples copied to the host.
int batch_chain_stats(fmc_batch* b, int chain, std::vector<double>& cs, std::vector<double>& gm,
                      std::vector<double>& ge) {
  const fmc::Batch& B = b->impl;
  const fmc::ChainDev& C = B.h_chains[chain];
  const fmc::InputDeck& d = B.sys_chains[B.chain_sys[chain]]->sys.deck;
  const int ng = (int)d.guests.size();
  cs.assign(1 + 14 * ng, 0.0);
  cs[0] = (double)C.prodcount;
  for (int g = 0; g < ng; g++)
    for (int k = 0; k < 6; k++) cs[1 + 14 * g + k] = C.stats[g][k];
  if (C.gasmol && C.prodcount > 0 && C.prodcount <= fmc::kSampleCap) {
    const size_t n = (size_t)ng * fmc::kSampleCap + 1;
    gm.resize(n);
    ge.resize(n);
    cudaSetDevice(B.device);
    cudaError_t e = cudaMemcpy(gm.data(), C.gasmol, sizeof(double) * n, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(ge.data(), C.gaseng, sizeof(double) * n, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) {
      fmc::set_last_error(cudaGetErrorString(e));
      return -100 - (int)e;
    }
  }
  return 0;
}
}  // namespace

int fmc_batch_write_numguests(fmc_batch* b, int chain, const void* trace, int nmoves, const char* outdir,
                              int append) {
  if (!b || chain < 0 || chain >= b->impl.nchains || !trace || nmoves < 0 || !outdir) {
    fmc::set_last_error("bad batch handle, chain index, trace or directory");
    return -1;
  }
  std::string err;
  int rc = b->impl.write_numguests(chain, static_cast<const fmc::MoveRecord*>(trace), nmoves, outdir, append != 0,
                                   err);
  if (rc) fmc::set_last_error(err);
  return rc;
}

int fmc_batch_pressures(fmc_batch* b, int chain, double* out) {
  if (!b || chain < 0 || chain >= b->impl.nchains || !out) {
    fmc::set_last_error("bad batch handle or chain index");
    return -1;
  }
  const fmc::Batch& B = b->impl;
  const int ng = (int)B.sys_chains[B.chain_sys[chain]]->sys.deck.guests.size();
  for (int i = 0; i < ng; i++) out[i] = B.h_chains[chain].press[i];
  out[ng] = B.h_chains[chain].despre;
  return 0;
}

int fmc_batch_window_stats(fmc_batch* b, int chain, double* out) {
  if (!b || chain < 0 || chain >= b->impl.nchains || !out) {
    fmc::set_last_error("bad batch handle or chain index");
    return -1;
  }
  const fmc::Batch& B = b->impl;
  const int ng = (int)B.sys_chains[B.chain_sys[chain]]->sys.deck.guests.size();
  fmc::window_stats_out(B.h_chains[chain].win, ng, out);
  return 0;
}

int fmc_batch_final_stats(fmc_batch* b, int chain, double* out) {
  if (!b || chain < 0 || chain >= b->impl.nchains || !out) {
    fmc::set_last_error("bad batch handle or chain index");
    return -1;
  }
  std::vector<double> cs, gm, ge;
  int rc = batch_chain_stats(b, chain, cs, gm, ge);
  if (rc) return rc;
  const fmc::Batch& B = b->impl;
  const fmc::ChainDev& C = B.h_chains[chain];
  fmc::final_stats((int)(cs.size() - 1) / 14, C.temp, cs.data(), C.win, gm.empty() ? nullptr : gm.data(),
                   ge.empty() ? nullptr : ge.data(), out);
  return 0;
}

int fmc_batch_write_report(fmc_batch* b, int chain, const char* path) {
  if (!b || chain < 0 || chain >= b->impl.nchains || !path) {
    fmc::set_last_error("bad batch handle, chain index or path");
    return -1;
  }
  const fmc::Batch& B = b->impl;
  const fmc::InputDeck& d = B.sys_chains[B.chain_sys[chain]]->sys.deck;
  std::vector<double> out(1 + 14 * d.guests.size());
  int rc = fmc_batch_final_stats(b, chain, out.data());
  if (rc) return rc;
  std::string err;
  rc = fmc::write_report(path, d, out.data(), B.h_chains[chain].win, B.h_chains[chain].temp, err);
  if (rc) fmc::set_last_error(err);
  return rc;
}

int fmc_batch_write_revive(fmc_batch* b, int chain, const char* outdir) {
  if (!b || chain < 0 || chain >= b->impl.nchains || !outdir) {
    fmc::set_last_error("bad batch handle, chain index or directory");
    return -1;
  }
  std::string err;
  int rc = b->impl.write_revive(chain, outdir, err);
  if (rc) fmc::set_last_error(err);
  return rc;
}

int fmc_batch_restart(fmc_batch* b, int chain, const char* revive_path) {
  if (!b || chain < 0 || chain >= b->impl.nchains || !revive_path) {
    fmc::set_last_error("bad batch handle, chain index or path");
    return -1;
  }
  std::string err;
  int rc = b->impl.restart(chain, revive_path, err);
  if (rc) fmc::set_last_error(err);
  return rc;
}

int fmc_batch_guest_coords(fmc_batch* b, int chain, int iguest, double* xyz, int* nmol, int* nsite) {
  if (!b || chain < 0 || chain >= b->impl.nchains) {
    fmc::set_last_error("bad batch handle or chain index");
    return -1;
  }
  const fmc::ChainDev& C = b->impl.h_chains[chain];
  const fmc::SysConst& Y = b->impl.h_sys[C.sys];
  if (iguest < 0 || iguest >= Y.nspecies) {
    fmc::set_last_error("species index out of range");
    return -1;
  }
  int ns = Y.sp[iguest].nsite, n = C.nmol[iguest];
  if (nmol) *nmol = n;
  if (nsite) *nsite = ns;
  if (xyz && n) {
    std::vector<double4> a(n * ns);
    cudaSetDevice(b->impl.device);
    cudaError_t e = cudaMemcpy(a.data(), C.gsite + C.seg_off[iguest], sizeof(double4) * n * ns, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) {
      fmc::set_last_error(cudaGetErrorString(e));
      return -100 - (int)e;
    }
    for (int i = 0; i < n * ns; i++) {
      xyz[3 * i] = a[i].x;
      xyz[3 * i + 1] = a[i].y;
      xyz[3 * i + 2] = a[i].z;
    }
  }
  return 0;
}

}  // extern "C"
