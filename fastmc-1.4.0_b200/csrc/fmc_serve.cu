// Serving: isotherm-point requests (a FastMC input deck + seed + budget) run as chains of
// the persistent batched kernel with continuous batching.  Each step admits queued requests
// into free slots while the device-memory budget allows (every slot holds its own framework
// system and chain state), advances every active slot by up to `moves` moves in one launch,
// and retires the chains that have used their budget (a move count, or with 0 the deck's own
// equilibration + production cycles), freeing their slots and memory for the next step.  The reference runs one such isotherm point per MPI rank (gcmc.f:334-417).
#include <cstring>
#include <deque>
#include <memory>
#include <string>
#include <vector>

#include "../../include/fastmc_b200.h"
#include "fmc_batch.h"

namespace fmc {
void set_last_error(const std::string& msg);

class Server {
 public:
  enum State { kQueued = 0, kRunning = 1, kDone = 2, kRejected = -1, kCancelled = -2 };
  struct Request {
    std::string dir;
    int seed[4];
    long long moves = 0;
    int state = kQueued, slot = -1;
    double result[32] = {0};
    std::string err;
  };
  struct Slot {
    int request = -1;
    std::unique_ptr<Chain> sys;
    std::vector<void*> allocs;
    size_t bytes = 0;
  };

  int device = 0;
  cudaStream_t st = nullptr;
  // phase tables in shared memory hold the old + new sites of one trial of up to
  // kServeMaxSites-site guests with kmax <= 32 per axis
  static constexpr int kServeMaxSites = 4;
  int nslots = 0, kcap = 0, tab_sites = 2 * kServeMaxSites, tab_stride = 0, smem = 0;
  size_t budget = 0, used = 0, slot_estimate = 64u << 20;
  int mixed = 0;
  long long recompute_every = 0;
  std::vector<Slot> slots;
  std::vector<Request> reqs;
  std::deque<int> queue;
  SysConst* h_sys = nullptr;
  SysConst* d_sys = nullptr;
  ChainDev* h_chains = nullptr;
  ChainDev* d_chains = nullptr;

  ~Server() {
    if (!st) return;
    cudaSetDevice(device);
    cudaStreamSynchronize(st);
    for (int i = 0; i < nslots; i++) release(i);
    if (d_sys) cudaFree(d_sys);
    if (d_chains) cudaFree(d_chains);
    if (h_sys) cudaFreeHost(h_sys);
    if (h_chains) cudaFreeHost(h_chains);
    cudaStreamDestroy(st);
  }

  int open(int n, int dev, size_t mem_budget, int k_cap, std::string& err) {
    device = dev;
    nslots = n;
    kcap = (k_cap + 3) & ~3;
    tab_stride = 3 * 32 + 3;  // kmax <= 32 per axis
    if (cudaSetDevice(dev) != cudaSuccess || cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) {
      err = "cannot select the device";
      return -100;
    }
    size_t free_b = 0, total_b = 0;
    cudaMemGetInfo(&free_b, &total_b);
    budget = mem_budget ? mem_budget : (size_t)(0.8 * (double)free_b);
    smem = batch_smem_bytes(kcap, tab_sites, tab_stride);
    if (smem > 220 * 1024) {
      err = "k-vector capacity exceeds the shared-memory budget of one CTA";
      return -9;
    }
    if (configure_batch_kernel(smem) != cudaSuccess) {
      err = "cannot configure the batched kernel";
      return -100;
    }
    slots.resize(n);
    cudaError_t e = cudaMallocHost(&h_sys, sizeof(SysConst) * n);
    if (e == cudaSuccess) e = cudaMallocHost(&h_chains, sizeof(ChainDev) * n);
    if (e == cudaSuccess) e = cudaMalloc(&d_sys, sizeof(SysConst) * n);
    if (e == cudaSuccess) e = cudaMalloc(&d_chains, sizeof(ChainDev) * n);
    if (e != cudaSuccess) {
      err = std::string("server allocation failed: ") + cudaGetErrorString(e);
      return -100 - (int)e;
    }
    std::memset(h_sys, 0, sizeof(SysConst) * n);
    std::memset(h_chains, 0, sizeof(ChainDev) * n);
    return 0;
  }

  int submit(const std::string& dir, const int* seed, long long moves) {
    Request r;
    r.dir = dir;
    std::memcpy(r.seed, seed, sizeof(r.seed));
    r.moves = moves;
    reqs.push_back(r);
    queue.push_back((int)reqs.size() - 1);
    return (int)reqs.size() - 1;
  }

  int cancel(int id) {
    if (id < 0 || id >= (int)reqs.size()) return -1;
    Request& r = reqs[id];
    if (r.state == kQueued) {
      for (auto it = queue.begin(); it != queue.end(); ++it)
        if (*it == id) {
          queue.erase(it);
          break;
        }
      r.state = kCancelled;
    } else if (r.state == kRunning) {
      snapshot(r.slot, r);
      release(r.slot);
      r.state = kCancelled;
    }
    return 0;
  }

  void release(int i) {
    Slot& s = slots[i];
    for (void* p : s.allocs) cudaFree(p);
    s.allocs.clear();
    s.sys.reset();
    used -= std::min(used, s.bytes);
    s.bytes = 0;
    s.request = -1;
    h_chains[i].active = 0;
  }

  void snapshot(int i, Request& r) {
    const ChainDev& C = h_chains[i];
    double* v = r.result;
    v[0] = (double)C.moves_done;
    v[1] = C.status;
    for (int g = 0; g < kMaxGuestTypes; g++) {
      v[2 + g] = C.nmol[g];
      v[6 + g] = C.energy[g];
    }
    v[10] = (double)C.prodcount;
    for (int k = 0; k < 5; k++) v[11 + k] = C.stats[0][k];
    v[16] = C.accept_ins;
    v[17] = C.accept_del;
    v[18] = (double)C.rechecks;
    v[19] = h_sys[i].S.K;
    v[20] = h_sys[i].S.nf;
    v[21] = C.temp;
    v[22] = C.press[0];
    v[23] = (double)r.moves;
    v[24] = C.lgchk ? 0.0 : 1.0;
    for (int k = 0; k < 5; k++) v[25 + k] = C.stats[1][k];
    v[30] = (double)C.gcmccount;
  }

  // Opens request `id` into free slot `i`; returns bytes used, or 0 (and marks the request
  // rejected) on failure.
  size_t admit(int id, int i) {
    Request& r = reqs[id];
    Slot& s = slots[i];
    size_t f0 = 0, f1 = 0, tot = 0;
    cudaMemGetInfo(&f0, &tot);
    std::string err;
    InputDeck deck;
    int rc = read_input_deck(r.dir, deck, err);
    if (!rc)
      for (auto& g : deck.guests)
        if (g.nmols) {
          rc = -8;
          err = "serving starts chains from an empty framework (NUMMOLS 0 for guests)";
        }
    if (!rc) {
      s.sys = std::make_unique<Chain>();
      rc = s.sys->open(r.dir, r.seed, device, err);
    }
    if (!rc && s.sys->sys.K > kcap) {
      rc = -9;
      err = "the request's k-vector count exceeds the server's capacity";
    }
    if (!rc && s.sys->sys.deck.kmax[0] + s.sys->sys.deck.kmax[1] + s.sys->sys.deck.kmax[2] + 3 > tab_stride) {
      rc = -9;
      err = "the request's kmax exceeds the server's phase-table capacity";
    }
    if (!rc)
      for (auto& g : deck.guests)
        if (g.nsite > kServeMaxSites) {
          rc = -9;
          err = "a guest of the request has more sites than the server's capacity";
        }
    int ts = 0;
    if (!rc) rc = make_sysconst(*s.sys, h_sys[i], s.allocs, &ts, err);
    if (!rc) rc = init_chain(deck, *s.sys, i, r.seed, h_chains[i], s.allocs, st, err);
    if (rc) {
      for (void* p : s.allocs) cudaFree(p);
      s.allocs.clear();
      s.sys.reset();
      std::memset(&h_chains[i], 0, sizeof(ChainDev));
      r.state = kRejected;
      r.err = err;
      r.result[1] = rc;
      return 0;
    }
    h_chains[i].budget = r.moves;
    cudaStreamSynchronize(st);
    cudaMemGetInfo(&f1, &tot);
    s.bytes = f0 > f1 ? f0 - f1 : 0;
    s.request = id;
    r.state = kRunning;
    r.slot = i;
    slot_estimate = std::max(slot_estimate, s.bytes);
    return s.bytes;
  }

  int step(int moves, int* n_active, int* n_queued, float* ms, std::string& err) {
    cudaSetDevice(device);
    // admission: FIFO, while a slot is free and the memory budget holds
    for (int i = 0; i < nslots && !queue.empty(); i++) {
      if (slots[i].request >= 0) continue;
      if (used + slot_estimate > budget) break;
      int id = queue.front();
      queue.pop_front();
      used += admit(id, i);
      if (reqs[id].state != kRunning) i--;  // slot still free
    }
    int active = 0;
    for (int i = 0; i < nslots; i++) active += slots[i].request >= 0;
    float t = 0.f;
    if (active) {
      cudaError_t e = cudaMemcpyAsync(d_sys, h_sys, sizeof(SysConst) * nslots, cudaMemcpyHostToDevice, st);
      if (e == cudaSuccess)
        e = cudaMemcpyAsync(d_chains, h_chains, sizeof(ChainDev) * nslots, cudaMemcpyHostToDevice, st);
      BatchLaunch L;
      std::memset(&L, 0, sizeof(L));
      L.chains = d_chains;
      L.systems = d_sys;
      L.nchains = nslots;
      L.moves = moves;
      L.kmax_smem = kcap;
      L.mixed = mixed;
      L.recompute_every = recompute_every;
      cudaEvent_t a, b;
      cudaEventCreate(&a);
      cudaEventCreate(&b);
      if (e == cudaSuccess) e = cudaEventRecord(a, st);
      if (e == cudaSuccess) e = launch_batch(L, smem, tab_stride, st);
      if (e == cudaSuccess) e = cudaEventRecord(b, st);
      if (e == cudaSuccess)
        e = cudaMemcpyAsync(h_chains, d_chains, sizeof(ChainDev) * nslots, cudaMemcpyDeviceToHost, st);
      if (e == cudaSuccess) e = cudaStreamSynchronize(st);
      if (e == cudaSuccess) cudaEventElapsedTime(&t, a, b);
      cudaEventDestroy(a);
      cudaEventDestroy(b);
      if (e != cudaSuccess) {
        err = std::string("serving launch failed: ") + cudaGetErrorString(e);
        return -100 - (int)e;
      }
    }
    // retirement
    for (int i = 0; i < nslots; i++) {
      int id = slots[i].request;
      if (id < 0) continue;
      const ChainDev& C = h_chains[i];
      if ((C.budget > 0 && C.moves_done >= C.budget) || !C.lgchk || C.status) {
        Request& r = reqs[id];
        snapshot(i, r);
        r.state = C.status ? kRejected : kDone;
        if (C.status) r.err = C.status == 75 ? "too many atoms in specified system" : "unsupported move drawn";
        release(i);
      }
    }
    if (n_active) *n_active = active;
    if (n_queued) *n_queued = (int)queue.size();
    if (ms) *ms = t;
    return 0;
  }
};

}  // namespace fmc

struct fmc_server {
  fmc::Server impl;
};

extern "C" {

int fmc_server_open(int slots, int device, long long mem_budget, int k_capacity, fmc_server** out) {
  if (!out || slots < 1 || k_capacity < 1 || mem_budget < 0) {
    fmc::set_last_error("bad server arguments");
    return -1;
  }
  fmc_server* s = new fmc_server();
  std::string err;
  int rc = s->impl.open(slots, device, (size_t)mem_budget, k_capacity, err);
  if (rc) {
    delete s;
    *out = nullptr;
    fmc::set_last_error(err);
    return rc;
  }
  *out = s;
  return 0;
}

void fmc_server_close(fmc_server* s) { delete s; }

int fmc_server_set_precision(fmc_server* s, int mixed, long long recompute_every) {
  if (!s || recompute_every < 0) {
    fmc::set_last_error("bad server handle or recompute interval");
    return -1;
  }
  s->impl.mixed = mixed & 7;
  s->impl.recompute_every = recompute_every;
  return 0;
}

int fmc_server_submit(fmc_server* s, const char* dir, const int* seed, long long moves, int* request_id) {
  if (!s || !dir || !seed || moves < 0 || !request_id) {
    fmc::set_last_error("bad submit arguments");
    return -1;
  }
  *request_id = s->impl.submit(dir, seed, moves);
  return 0;
}

int fmc_server_cancel(fmc_server* s, int request_id) {
  if (!s || s->impl.cancel(request_id)) {
    fmc::set_last_error("bad server handle or request id");
    return -1;
  }
  return 0;
}

int fmc_server_step(fmc_server* s, int moves, int* active, int* queued, float* device_ms) {
  if (!s || moves < 1) {
    fmc::set_last_error("bad server handle or move count");
    return -1;
  }
  std::string err;
  int rc = s->impl.step(moves, active, queued, device_ms, err);
  if (rc) fmc::set_last_error(err);
  return rc;
}

int fmc_server_poll(fmc_server* s, int request_id, int* state, double* out) {
  if (!s || request_id < 0 || request_id >= (int)s->impl.reqs.size()) {
    fmc::set_last_error("bad server handle or request id");
    return -1;
  }
  const fmc::Server::Request& r = s->impl.reqs[request_id];
  if (state) *state = r.state;
  if (out) std::memcpy(out, r.result, sizeof(r.result));
  if (r.state == fmc::Server::kRejected) fmc::set_last_error(r.err);
  return 0;
}

int fmc_server_memory(fmc_server* s, long long* used, long long* budget) {
  if (!s) {
    fmc::set_last_error("bad server handle");
    return -1;
  }
  if (used) *used = (long long)s->impl.used;
  if (budget) *budget = (long long)s->impl.budget;
  return 0;
}

}  // extern "C"
