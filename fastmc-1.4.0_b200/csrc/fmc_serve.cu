// Serving: isotherm-point requests (a FastMC input deck + seed + budget) run as chains of
// the persistent batched kernel with continuous batching.  Host worker threads parse each
// queued request's deck and build its host tables ahead of time; each step admits prepared
// requests from the front of the queue into free slots while the device-memory budget allows
// (every slot holds its own framework system and chain state), advances every active slot by
// up to `moves` moves in one launch, and retires the chains that have used their budget (a
// move count, or with 0 the deck's own equilibration + production cycles), freeing their
// slots and memory for the next step.  The reference runs one such isotherm point per MPI
// rank (gcmc.f:334-417).
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/fastmc_b200.h"
#include "fmc_batch.h"

namespace fmc {
void set_last_error(const std::string& msg);

namespace {
double now_ms() {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}
}  // namespace

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
    // host preparation (worker threads): 0 pending, 1 ready
    std::atomic<int> prepared{0};
    int prep_rc = 0;
    std::string prep_err;
    std::unique_ptr<HostSystem> host;
    size_t bytes_estimate = 0;
  };
  struct Slot {
    int request = -1;
    SlotMemory mem;
    long long vox_cap = 0;  // voxel-list entries allocated
    bool fresh = false;     // admitted in this step; capacity not checked yet
  };

  // phase tables in shared memory hold the old + new sites of one trial of up to
  // kServeMaxSites-site guests with kmax <= 32 per axis
  static constexpr int kServeMaxSites = 4;
  int device = 0;
  cudaStream_t st = nullptr;
  int nslots = 0, kcap = 0, tab_sites = 2 * kServeMaxSites, tab_stride = 0, smem = 0;
  size_t budget = 0, used = 0;
  cudaMemPool_t pool = nullptr;
  int mixed = 0;
  long long recompute_every = 0;
  std::vector<Slot> slots;
  std::vector<std::unique_ptr<Request>> reqs;  // the vector is guarded by mu; entries are stable
  std::deque<int> queue;                       // admission order (caller's thread only)
  SysConst* h_sys = nullptr;
  SysConst* d_sys = nullptr;
  ChainDev* h_chains = nullptr;
  ChainDev* d_chains = nullptr;
  ChainDev* h_out = nullptr;      // pinned: control blocks as the last launch left them
  int* h_vox_total = nullptr;     // pinned: exact voxel-list size of each slot's last build
  std::vector<char> launched;     // slots in the current launch
  cudaStream_t st2 = nullptr;     // admission stream (slot set-up beside the running launch)
  Staging stage;                  // pinned staging of slot uploads
  cudaEvent_t ev0 = nullptr, ev1 = nullptr, ev_h2d = nullptr;
  // worker pool
  std::mutex mu;
  std::condition_variable cv;
  std::deque<int> prep_queue;
  std::vector<std::thread> workers;
  bool stopping = false;
  // accounting
  long long admitted = 0, retired = 0, launches = 0, moves_run = 0, last_moves = 0;
  double admit_ms = 0, launch_ms = 0, wait_ms = 0;
  std::atomic<long long> prep_us{0};

  ~Server() {
    {
      std::lock_guard<std::mutex> lk(mu);
      stopping = true;
    }
    cv.notify_all();
    for (auto& t : workers) t.join();
    if (!st) return;
    cudaSetDevice(device);
    cudaStreamSynchronize(st);
    if (st2) cudaStreamSynchronize(st2);
    for (int i = 0; i < nslots; i++) release(i);
    if (st2) cudaStreamSynchronize(st2);
    if (pool) cudaMemPoolDestroy(pool);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (ev_h2d) cudaEventDestroy(ev_h2d);
    if (h_out) cudaFreeHost(h_out);
    if (h_vox_total) cudaFreeHost(h_vox_total);
    if (stage.base) cudaFreeHost(stage.base);
    if (st2) cudaStreamDestroy(st2);
    if (d_sys) cudaFree(d_sys);
    if (d_chains) cudaFree(d_chains);
    if (h_sys) cudaFreeHost(h_sys);
    if (h_chains) cudaFreeHost(h_chains);
    cudaStreamDestroy(st);
  }

  int open(int n, int dev, size_t mem_budget, int k_cap, int nworkers, std::string& err) {
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
    if (configure_batch_kernel(smem) != cudaSuccess || configure_kernels() != cudaSuccess ||
        configure_recip_kernels() != cudaSuccess) {
      err = "cannot configure the kernels";
      return -100;
    }
    // slot memory: a pool of its own that keeps freed blocks for the next admissions
    cudaMemPoolProps props;
    std::memset(&props, 0, sizeof(props));
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    if (cudaMemPoolCreate(&pool, &props) != cudaSuccess) {
      err = "cannot create the slot memory pool";
      return -100;
    }
    unsigned long long keep = ~0ull;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    if (cudaStreamCreateWithFlags(&st2, cudaStreamNonBlocking) != cudaSuccess) {
      err = "cannot create the admission stream";
      return -100;
    }
    slots.resize(n);
    launched.assign(n, 0);
    for (auto& sl : slots) {
      sl.mem.st = st2;
      sl.mem.pool = pool;
    }
    stage.cap = 64u << 20;
    cudaError_t e = cudaMallocHost(&stage.base, stage.cap);
    if (e == cudaSuccess) e = cudaMallocHost(&h_out, sizeof(ChainDev) * n);
    if (e == cudaSuccess) e = cudaMallocHost(&h_vox_total, sizeof(int) * n);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ev_h2d, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaMallocHost(&h_sys, sizeof(SysConst) * n);
    if (e == cudaSuccess) e = cudaMallocHost(&h_chains, sizeof(ChainDev) * n);
    if (e == cudaSuccess) e = cudaMalloc(&d_sys, sizeof(SysConst) * n);
    if (e == cudaSuccess) e = cudaMalloc(&d_chains, sizeof(ChainDev) * n);
    if (e == cudaSuccess) e = cudaEventCreate(&ev0);
    if (e == cudaSuccess) e = cudaEventCreate(&ev1);
    if (e != cudaSuccess) {
      err = std::string("server allocation failed: ") + cudaGetErrorString(e);
      return -100 - (int)e;
    }
    std::memset(h_sys, 0, sizeof(SysConst) * n);
    std::memset(h_chains, 0, sizeof(ChainDev) * n);
    for (int w = 0; w < nworkers; w++) workers.emplace_back([this] { worker(); });
    return 0;
  }

  // Host preparation of one request: deck, host tables and the serving capacity checks.
  void prepare(Request& r) {
    const double t0 = now_ms();
    auto h = std::make_unique<HostSystem>();
    std::string err;
    int rc = prepare_system(r.dir, *h, err);
    if (!rc)
      for (auto& g : h->deck.guests)
        if (g.nmols) {
          rc = -8;
          err = "serving starts chains from an empty framework (NUMMOLS 0 for guests)";
        }
    if (!rc && h->K > kcap) {
      rc = -9;
      err = "the request's k-vector count exceeds the server's capacity";
    }
    if (!rc && h->deck.kmax[0] + h->deck.kmax[1] + h->deck.kmax[2] + 3 > tab_stride) {
      rc = -9;
      err = "the request's kmax exceeds the server's phase-table capacity";
    }
    if (!rc)
      for (auto& g : h->deck.guests)
        if (g.nsite > kServeMaxSites) {
          rc = -9;
          err = "a guest of the request has more sites than the server's capacity";
        }
    r.prep_rc = rc;
    r.prep_err = err;
    if (!rc) {
      r.bytes_estimate = slot_bytes_estimate(*h);
      r.host = std::move(h);
    }
    prep_us += (long long)((now_ms() - t0) * 1000.0);
    r.prepared.store(1, std::memory_order_release);
  }

  // Worker threads: host preparation of queued requests, in submission order.
  void worker() {
    for (;;) {
      Request* r = nullptr;
      {
        std::unique_lock<std::mutex> lk(mu);
        cv.wait(lk, [this] { return stopping || !prep_queue.empty(); });
        if (stopping) return;
        r = reqs[prep_queue.front()].get();
        prep_queue.pop_front();
      }
      prepare(*r);
    }
  }

  Request& req(int id) {
    std::lock_guard<std::mutex> lk(mu);
    return *reqs[id];
  }

  int nreqs() {
    std::lock_guard<std::mutex> lk(mu);
    return (int)reqs.size();
  }

  int submit(const std::string& dir, const int* seed, long long moves) {
    auto r = std::make_unique<Request>();
    r->dir = dir;
    std::memcpy(r->seed, seed, sizeof(r->seed));
    r->moves = moves;
    int id;
    {
      std::lock_guard<std::mutex> lk(mu);
      reqs.push_back(std::move(r));
      id = (int)reqs.size() - 1;
      if (!workers.empty()) prep_queue.push_back(id);
    }
    cv.notify_one();
    queue.push_back(id);
    return id;
  }

  int cancel(int id) {
    if (id < 0 || id >= nreqs()) return -1;
    Request& r = req(id);
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
    used -= std::min(used, s.mem.bytes);
    s.mem.release();
    s.request = -1;
    h_chains[i].active = 0;
  }

  // Device bytes of a slot for admission: voxel entries from the framework's mean density
  // (+15%), plus atoms, tables, k-vector tables and guest segments.
  static size_t slot_bytes_estimate(const HostSystem& h) {
    const double lim = std::sqrt(h.vox_lim2);
    const double per_vox = std::min((double)h.nf, h.nf * (4.0 / 3.0 * kPi * lim * lim * lim) / h.cell.volm);
    const double nv = (double)h.nvox[0] * h.nvox[1] * h.nvox[2];
    double b = 1.15 * nv * per_vox * (sizeof(double4) + 1) + 4.0 * (nv + 1) + 36.0 * h.nf;
    b += 12.0 * (h.erc.size() + h.vvv.size()) + 4.0 * h.pair_row.size() + 60.0 * h.K;
    b += 36.0 * h.deck.maxguest * h.deck.guests.size();
    b += 2.0 * 8.0 * ((double)kSampleCap * h.deck.guests.size() + 1);  // stored production samples
    return (size_t)b + (64u << 10);
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

  void reject(Request& r, int rc, const std::string& err) {
    r.state = kRejected;
    r.err = err;
    r.result[1] = rc;
    r.host.reset();
  }

  // Enqueues the slot set-up of prepared request `id` into free slot `i` on the admission
  // stream; returns the slot's device bytes, or 0 (and marks the request rejected).
  size_t admit(int id, int i) {
    Request& r = req(id);
    Slot& s = slots[i];
    if (r.prep_rc) {
      reject(r, r.prep_rc, r.prep_err);
      return 0;
    }
    const size_t need = slot_staging_bytes(*r.host);
    if (stage.used + need > stage.cap) {  // the staged bytes of earlier admissions are read by now
      cudaStreamSynchronize(st2);
      stage.used = 0;
      if (need > stage.cap) {
        cudaFreeHost(stage.base);
        stage.cap = need;
        if (cudaMallocHost(&stage.base, stage.cap) != cudaSuccess) {
          stage.base = nullptr;
          stage.cap = 0;
        }
      }
    }
    std::string err;
    s.vox_cap = slot_voxel_capacity(*r.host);
    int rc = build_slot(*r.host, i, r.seed, s.mem, stage, s.vox_cap, &h_vox_total[i], h_sys[i], h_chains[i], err);
    if (rc) {
      s.mem.release();
      std::memset(&h_chains[i], 0, sizeof(ChainDev));
      reject(r, rc, err);
      return 0;
    }
    h_chains[i].budget = r.moves;
    s.request = id;
    s.fresh = true;
    r.state = kRunning;
    r.slot = i;
    admitted++;
    return s.mem.bytes;
  }

  // Admission: FIFO, while a slot is free, the front request is prepared and the memory budget
  // holds.  With nothing running, waits for the front request's preparation.
  void admit_queued(int running) {
    const double t0 = now_ms();
    for (int i = 0; i < nslots && !queue.empty(); i++) {
      if (slots[i].request >= 0) continue;
      const int id = queue.front();
      Request& r = req(id);
      if (workers.empty()) {
        prepare(r);
      } else if (!r.prepared.load(std::memory_order_acquire)) {
        if (running) break;
        const double w0 = now_ms();
        while (!r.prepared.load(std::memory_order_acquire)) std::this_thread::sleep_for(std::chrono::microseconds(200));
        wait_ms += now_ms() - w0;
      }
      if (!r.prep_rc && used + r.bytes_estimate > budget) {
        if (r.bytes_estimate > budget) {
          queue.pop_front();
          reject(r, -10, "the request's device footprint exceeds the server's memory budget");
          i--;
          continue;
        }
        break;  // wait for retirements
      }
      queue.pop_front();
      used += admit(id, i);
      if (r.state != kRunning) i--;  // slot still free
    }
    admit_ms += now_ms() - t0;
  }

  // Once the admission stream has drained: slots whose voxel lists outgrew the estimate are
  // rebuilt at their exact size (rare; the estimate carries 15% headroom).
  int settle_admissions(std::string& err) {
    cudaError_t e = cudaStreamSynchronize(st2);
    if (e != cudaSuccess) {
      err = std::string("slot set-up failed: ") + cudaGetErrorString(e);
      return -100 - (int)e;
    }
    stage.used = 0;
    for (int i = 0; i < nslots; i++) {
      Slot& s = slots[i];
      if (s.request < 0 || !s.fresh) continue;
      s.fresh = false;
      Request& r = req(s.request);
      if ((long long)h_vox_total[i] > s.vox_cap) {
        used -= std::min(used, s.mem.bytes);
        s.mem.release();
        s.vox_cap = h_vox_total[i];
        std::string e2;
        int rc = build_slot(*r.host, i, r.seed, s.mem, stage, s.vox_cap, &h_vox_total[i], h_sys[i], h_chains[i], e2);
        if (rc == 0 && cudaStreamSynchronize(st2) != cudaSuccess) rc = -100;
        stage.used = 0;
        if (rc || (long long)h_vox_total[i] > s.vox_cap) {
          s.mem.release();
          s.request = -1;
          std::memset(&h_chains[i], 0, sizeof(ChainDev));
          reject(r, rc ? rc : -12, rc ? e2 : "voxel lists changed size between builds");
          continue;
        }
        h_chains[i].budget = r.moves;
        used += s.mem.bytes;
      }
      r.host.reset();
    }
    return 0;
  }

  int step(int moves, int* n_active, int* n_queued, float* ms, std::string& err) {
    cudaSetDevice(device);
    int running = 0;
    for (int i = 0; i < nslots; i++) {
      launched[i] = slots[i].request >= 0;
      running += launched[i];
    }
    if (!running) {  // nothing on the device: admit first, then launch what was admitted
      admit_queued(0);
      int rc = settle_admissions(err);
      if (rc) return rc;
      for (int i = 0; i < nslots; i++) {
        launched[i] = slots[i].request >= 0;
        running += launched[i];
      }
    }
    float t = 0.f;
    last_moves = 0;
    cudaError_t e = cudaSuccess;
    if (running) {
      e = cudaMemcpyAsync(d_sys, h_sys, sizeof(SysConst) * nslots, cudaMemcpyHostToDevice, st);
      if (e == cudaSuccess)
        e = cudaMemcpyAsync(d_chains, h_chains, sizeof(ChainDev) * nslots, cudaMemcpyHostToDevice, st);
      if (e == cudaSuccess) e = cudaEventRecord(ev_h2d, st);
      BatchLaunch L;
      std::memset(&L, 0, sizeof(L));
      L.chains = d_chains;
      L.systems = d_sys;
      L.nchains = nslots;
      L.moves = moves;
      L.kmax_smem = kcap;
      L.mixed = mixed;
      L.recompute_every = recompute_every;
      if (e == cudaSuccess) e = cudaEventRecord(ev0, st);
      if (e == cudaSuccess) e = launch_batch(L, smem, tab_stride, st);
      if (e == cudaSuccess) e = cudaEventRecord(ev1, st);
      if (e == cudaSuccess)
        e = cudaMemcpyAsync(h_out, d_chains, sizeof(ChainDev) * nslots, cudaMemcpyDeviceToHost, st);
      // requests admitted now set up on the admission stream while the launch runs; their host
      // control blocks change only after the launch's copy of them has been read
      if (e == cudaSuccess) e = cudaEventSynchronize(ev_h2d);
      if (e == cudaSuccess) admit_queued(running);
      if (e == cudaSuccess) e = cudaStreamSynchronize(st);
      if (e == cudaSuccess) cudaEventElapsedTime(&t, ev0, ev1);
      if (e != cudaSuccess) {
        err = std::string("serving launch failed: ") + cudaGetErrorString(e);
        return -100 - (int)e;
      }
      int rc = settle_admissions(err);
      if (rc) return rc;
      launches++;
      launch_ms += t;
      for (int i = 0; i < nslots; i++)
        if (launched[i]) {
          last_moves += h_out[i].moves_done - h_chains[i].moves_done;
          h_chains[i] = h_out[i];
        }
      moves_run += last_moves;
    }
    // retirement of the chains that ran
    for (int i = 0; i < nslots; i++) {
      int id = slots[i].request;
      if (id < 0 || !launched[i]) continue;
      const ChainDev& C = h_chains[i];
      if ((C.budget > 0 && C.moves_done >= C.budget) || !C.lgchk || C.status) {
        Request& r = req(id);
        snapshot(i, r);
        r.state = C.status ? kRejected : kDone;
        if (C.status) r.err = C.status == 75 ? "too many atoms in specified system" : "chain stopped with an unknown status";
        release(i);
        retired++;
      }
    }
    if (n_active) *n_active = running;
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
  unsigned hw = std::thread::hardware_concurrency();
  int nworkers = (int)std::max(1u, std::min(8u, hw > 1 ? hw - 1 : 1u));
  int rc = s->impl.open(slots, device, (size_t)mem_budget, k_capacity, nworkers, err);
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
  if (!s || request_id < 0 || request_id >= s->impl.nreqs()) {
    fmc::set_last_error("bad server handle or request id");
    return -1;
  }
  const fmc::Server::Request& r = s->impl.req(request_id);
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

int fmc_server_stats(fmc_server* s, double* out) {
  if (!s || !out) {
    fmc::set_last_error("bad server handle");
    return -1;
  }
  const fmc::Server& v = s->impl;
  out[0] = (double)v.admitted;
  out[1] = (double)v.retired;
  out[2] = (double)v.launches;
  out[3] = v.admit_ms;
  out[4] = v.launch_ms;
  out[5] = v.wait_ms;
  out[6] = (double)v.prep_us.load() / 1000.0;
  out[7] = (double)v.workers.size();
  out[8] = (double)v.moves_run;
  out[9] = (double)v.last_moves;
  return 0;
}

}  // extern "C"
