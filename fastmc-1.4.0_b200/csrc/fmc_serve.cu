// Serving: isotherm-point requests (a FastMC input deck + seed + budget) run as chains of
// the persistent batched kernel with continuous batching.  Host worker threads parse each
// queued request's deck and build its host tables ahead of time.  Launches are pipelined: a
// step queues the next launch of every running slot (the device keeps each chain's control
// block between launches) and only then completes the previous launch: it retires the chains
// that used their budget (a move count, or with 0 the deck's own equilibration + production
// cycles; a finished chain marks itself inactive, so the launch already queued skips it) and
// admits prepared requests from the front of the queue into free slots while the device-memory
// budget allows.  Worker threads enqueue each request's device slot on their own streams ahead
// of admission without waiting for it (an event marks the build's end), so a worker goes on to
// the next deck while the device builds; admission installs a slot whose build has completed,
// or builds one on a second stream beside the running launch for the launch after it.  So
// launches follow one another without waiting for the host.  The reference runs one such
// isotherm point per MPI rank (gcmc.f:334-417).
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
#include "fmc_restart.h"

namespace fmc {
void set_last_error(const std::string& msg);

namespace {
double now_ms() {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}
}  // namespace

// A slot built ahead by a worker: its build is enqueued on the worker's stream and `done` is
// recorded after it; *vox_total (pinned) receives the exact voxel-list size, checked against
// vox_cap once `done` has completed.
struct Prebuilt {
  SlotMemory mem;
  SysConst Y;
  ChainDev C;
  long long vox_cap = 0;
  cudaEvent_t done = nullptr;
  int word = -1;  // index of vox_total in the server's pinned words
  int* vox_total = nullptr;
};

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
    std::unique_ptr<SlotStart> start;  // null: the empty framework
    // the chain's state when it finished (kept while keep_final is on): guest sites per species
    // (x, y, z molecule-major), the production flag, chainstats, energies and the last energy
    // change, what a REVIVE / REVCON holds
    struct Final {
      std::vector<std::vector<double>> xyz;
      bool production = false;
      std::vector<double> chainstats, energy;
      double last_dE = 0.0;
    };
    std::unique_ptr<Final> fin;
    size_t bytes_estimate = 0;
    // the device slot a worker built ahead of admission (null: built at admission instead)
    std::unique_ptr<struct Prebuilt> pre;
  };
  // A worker's own stream and a ring of pinned staging buffers for building slots ahead: a
  // buffer is reused once the build that read it has completed (its event).
  static constexpr int kRing = 4;
  struct WorkerRes {
    cudaStream_t st = nullptr;
    Staging stage[kRing];
    cudaEvent_t stage_done[kRing] = {};
    bool stage_busy[kRing] = {};
    int next = 0;
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
  size_t budget = 0;
  std::atomic<size_t> used{0};      // device bytes of admitted slots
  size_t prebuilt_bytes = 0;        // device bytes of slots built ahead (guarded by mu)
  int prebuilt_count = 0;
  int building = 0;                 // slots being built ahead right now (guarded by mu)
  static constexpr int kMaxPrebuilt = 64;  // slots built ahead at most
  std::vector<WorkerRes> wres;
  int* h_words = nullptr;           // pinned voxel-list sizes of slots built ahead
  std::vector<int> free_words;      // (guarded by mu)
  cudaMemPool_t pool = nullptr;
  std::vector<Slot> slots;
  std::vector<std::unique_ptr<Request>> reqs;  // the vector is guarded by mu; entries are stable
  std::deque<int> queue;                       // admission order (caller's thread only)
  SysConst* h_sys = nullptr;
  SysConst* d_sys = nullptr;
  ChainDev* h_chains = nullptr;   // pinned: each slot's control block as of the last completed launch
  ChainDev* d_chains = nullptr;   // the device copy the launches read and write
  ChainDev* h_out[2] = {nullptr, nullptr};  // pinned: control blocks after launch buffer b
  int* h_vox_total = nullptr;     // pinned: exact voxel-list size of each slot's last build
  std::vector<int> launched[2];   // per slot, the request launch buffer b ran (-1: none)
  int* h_zero = nullptr;          // pinned 0: the `active` flag of a cancelled slot
  int inflight = -1;              // buffer of the launch queued and not yet completed (-1: none)
  int next_buf = 0;
  std::vector<int> fresh;         // slots admitted since the last launch (uploaded before the next)
  std::vector<int> deactivate;    // cancelled slots to switch off on the device before the next launch
  std::vector<std::pair<int, int>> deferred;  // (slot, buffer): memory freed once that launch completed
  std::vector<int> done_log;      // requests that reached a final state, for poll_done
  std::vector<int> cancelled_unprepared;  // cancelled while a worker prepared them (caller's thread only)
  cudaStream_t st2 = nullptr;     // admission stream (slot set-up beside the running launch)
  Staging stage;                  // pinned staging of slot uploads
  cudaEvent_t ev_start[2] = {nullptr, nullptr}, ev_end[2] = {nullptr, nullptr}, ev_done[2] = {nullptr, nullptr};
  cudaEvent_t ev_admit = nullptr;  // recorded on the admission stream after the last admission
  // worker pool
  std::mutex mu;
  std::condition_variable cv;
  std::deque<int> prep_queue;
  std::vector<std::thread> workers;
  bool stopping = false;
  // accounting
  long long admitted = 0, retired = 0, launches = 0, moves_run = 0, last_moves = 0;
  double admit_ms = 0, launch_ms = 0, wait_ms = 0;
  std::atomic<long long> prep_us{0}, prep_host_us{0}, prep_dev_us{0};
  std::atomic<double> voxel_edge{2.0};  // neighbour-list voxel edge (A) of requests prepared from now on
  long long admit_prebuilt = 0, admit_built = 0;
  bool keep_final = false;         // copy a finished chain's guests to the host before its slot is freed
  cudaStream_t st3 = nullptr;      // those copies (created when keep_final is first turned on)

  ~Server() {
    {
      std::lock_guard<std::mutex> lk(mu);
      stopping = true;
    }
    cv.notify_all();
    for (auto& t : workers) t.join();
    if (!st) return;
    cudaSetDevice(device);
    for (auto& r : reqs)
      if (r->pre) {
        r->pre->mem.release();
        if (r->pre->done) cudaEventDestroy(r->pre->done);
        r->pre.reset();
      }
    cudaStreamSynchronize(st);
    if (st2) cudaStreamSynchronize(st2);
    for (int i = 0; i < nslots; i++) release(i);  // frees on the slot's stream (st2 or a worker's)
    if (st2) cudaStreamSynchronize(st2);
    for (WorkerRes& w : wres) {
      if (w.st) cudaStreamSynchronize(w.st);
      for (int k = 0; k < kRing; k++) {
        if (w.stage[k].base) cudaFreeHost(w.stage[k].base);
        if (w.stage_done[k]) cudaEventDestroy(w.stage_done[k]);
      }
      if (w.st) cudaStreamDestroy(w.st);
    }
    if (h_words) cudaFreeHost(h_words);
    if (pool) cudaMemPoolDestroy(pool);
    for (int b = 0; b < 2; b++) {
      if (ev_start[b]) cudaEventDestroy(ev_start[b]);
      if (ev_end[b]) cudaEventDestroy(ev_end[b]);
      if (ev_done[b]) cudaEventDestroy(ev_done[b]);
      if (h_out[b]) cudaFreeHost(h_out[b]);
    }
    if (ev_admit) cudaEventDestroy(ev_admit);
    if (h_vox_total) cudaFreeHost(h_vox_total);
    if (h_zero) cudaFreeHost(h_zero);
    if (stage.base) cudaFreeHost(stage.base);
    if (st2) cudaStreamDestroy(st2);
    if (st3) cudaStreamDestroy(st3);
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
    launched[0].assign(n, -1);
    launched[1].assign(n, -1);
    for (auto& sl : slots) {
      sl.mem.st = st2;
      sl.mem.pool = pool;
    }
    stage.cap = 64u << 20;
    cudaError_t e = cudaMallocHost(&stage.base, stage.cap);
    for (int b = 0; b < 2 && e == cudaSuccess; b++) {
      e = cudaMallocHost(&h_out[b], sizeof(ChainDev) * n);
      if (e == cudaSuccess) e = cudaEventCreate(&ev_start[b]);
      if (e == cudaSuccess) e = cudaEventCreate(&ev_end[b]);
      if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ev_done[b], cudaEventDisableTiming);
    }
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ev_admit, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaMallocHost(&h_vox_total, sizeof(int) * n);
    if (e == cudaSuccess) e = cudaMallocHost(&h_zero, sizeof(int));
    if (e == cudaSuccess) *h_zero = 0;
    if (e == cudaSuccess) e = cudaMallocHost(&h_sys, sizeof(SysConst) * n);
    if (e == cudaSuccess) e = cudaMallocHost(&h_chains, sizeof(ChainDev) * n);
    if (e == cudaSuccess) e = cudaMalloc(&d_sys, sizeof(SysConst) * n);
    if (e == cudaSuccess) e = cudaMalloc(&d_chains, sizeof(ChainDev) * n);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_chains, 0, sizeof(ChainDev) * n, st);  // every slot inactive
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
      err = std::string("server allocation failed: ") + cudaGetErrorString(e);
      return -100 - (int)e;
    }
    std::memset(h_sys, 0, sizeof(SysConst) * n);
    std::memset(h_chains, 0, sizeof(ChainDev) * n);
    wres.resize(nworkers);
    for (WorkerRes& w : wres) {
      if (cudaStreamCreateWithFlags(&w.st, cudaStreamNonBlocking) != cudaSuccess) {
        err = "cannot create a worker's stream";
        return -100;
      }
      for (int k = 0; k < kRing; k++) {
        w.stage[k].cap = 4u << 20;
        if (cudaMallocHost(&w.stage[k].base, w.stage[k].cap) != cudaSuccess ||
            cudaEventCreateWithFlags(&w.stage_done[k], cudaEventDisableTiming) != cudaSuccess) {
          err = "cannot allocate a worker's staging buffers";
          return -100;
        }
      }
    }
    if (cudaMallocHost(&h_words, sizeof(int) * kMaxPrebuilt) != cudaSuccess) {
      err = "cannot allocate the pinned voxel-size words";
      return -100;
    }
    for (int k = kMaxPrebuilt - 1; k >= 0; k--) free_words.push_back(k);
    for (int w = 0; w < nworkers; w++) workers.emplace_back([this, w] { worker(w); });
    return 0;
  }

  // Host preparation of one request: deck, host tables and the serving capacity checks.
  void prepare(Request& r, WorkerRes* w = nullptr) {
    const double t0 = now_ms();
    auto h = std::make_unique<HostSystem>();
    std::string err;
    int rc = prepare_system(r.dir, *h, err, voxel_edge.load());
    std::string revive;  // CONTROL `restart`: the REVIVE of branch01 beside the deck, if any
    if (!rc && h->deck.lrestart && !h->deck.lspe) {
      BranchChoice b;
      rc = choose_branch(r.dir, 0, b, err);
      revive = b.revive;
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
    bool preloaded = false;
    for (auto& g : h->deck.guests) preloaded = preloaded || g.nmols > 0;
    if (!rc && (preloaded || !revive.empty())) rc = start_state(r, revive, err);
    r.prep_rc = rc;
    r.prep_err = err;
    const double t1 = now_ms();
    prep_host_us += (long long)((t1 - t0) * 1000.0);
    if (!rc) {
      r.bytes_estimate = slot_bytes_estimate(*h);
      r.host = std::move(h);
      if (w) {
        prebuild(r, *w);
        prep_dev_us += (long long)((now_ms() - t1) * 1000.0);
      }
    }
    prep_us += (long long)((now_ms() - t0) * 1000.0);
    r.prepared.store(1, std::memory_order_release);
  }

  // The state a request with guests starts from (the deck's preloaded guests, or the REVIVE of
  // its CONTROL `restart`): a plain chain opened on the deck at the server's voxel edge computes
  // the single point and S(k) of every atom on the device, as the batched path's own chain
  // does; its results and guest sites are kept in host memory and the chain is closed.
  int start_state(Request& r, const std::string& revive, std::string& err) {
    Chain ch;
    int rc = ch.open(r.dir, r.seed, device, err, voxel_edge.load());
    Revive rv;
    if (!rc && !revive.empty()) rc = read_revive(revive, ch.sys.deck, rv, err);
    if (!rc && !revive.empty()) rc = ch.restart(rv, err);
    if (rc) return rc;
    auto S = std::make_unique<SlotStart>();
    const InputDeck& d = ch.sys.deck;
    S->sk.resize(ch.sys.K);
    cudaError_t e = cudaStreamSynchronize(ch.st);
    if (e == cudaSuccess && ch.sys.K)
      e = cudaMemcpy(S->sk.data(), ch.sk, sizeof(double2) * ch.sys.K, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) {
      err = std::string("start state read-back failed: ") + cudaGetErrorString(e);
      return -100 - (int)e;
    }
    S->spenergy = ch.spenergy;
    for (size_t g = 0; g < ch.sp.size(); g++) {
      const GuestSpecies& G = d.guests[g];
      const int n = ch.sp[g].nmol * G.nsite;
      S->nmol.push_back(ch.sp[g].nmol);
      S->sites.emplace_back(n);
      S->types.emplace_back(n);
      for (int i = 0; i < n; i++) {
        const double* x = &ch.sp[g].xyz[3 * i];
        S->sites[g][i] = make_double4(x[0], x[1], x[2], G.charge[i % G.nsite]);
        S->types[g][i] = G.type[i % G.nsite];
      }
    }
    if (!revive.empty()) {
      S->from_revive = true;
      S->production = rv.production;
      S->chainstats = rv.chainstats;
      if ((int)S->chainstats.size() != 1 + 14 * (int)d.guests.size()) S->chainstats.assign(1 + 14 * d.guests.size(), 0.0);
    }
    r.start = std::move(S);
    return 0;
  }

  // A worker enqueues the request's device slot on its own stream, while the memory budget
  // allows, and records an event after it without waiting: admission installs the slot once
  // the event has completed and the voxel lists have been checked against their estimate.  On
  // any failure the slot is left to be built at admission.
  void prebuild(Request& r, WorkerRes& w) {
    int word = -1;
    {
      std::lock_guard<std::mutex> lk(mu);
      if (prebuilt_count >= kMaxPrebuilt || free_words.empty() ||
          used.load() + prebuilt_bytes + r.bytes_estimate > budget)
        return;
      prebuilt_bytes += r.bytes_estimate;
      prebuilt_count++;
      building++;
      word = free_words.back();
      free_words.pop_back();
    }
    auto P = std::make_unique<Prebuilt>();
    P->mem.st = w.st;
    P->mem.pool = pool;
    P->word = word;
    P->vox_total = h_words + word;
    *P->vox_total = 0;
    const int k = w.next;
    w.next = (w.next + 1) % kRing;
    Staging& sg = w.stage[k];
    bool ok = !w.stage_busy[k] || cudaEventSynchronize(w.stage_done[k]) == cudaSuccess;  // read by now
    const size_t need = slot_staging_bytes(*r.host);
    if (ok && need > sg.cap) {
      cudaFreeHost(sg.base);
      sg.cap = need;
      if (cudaMallocHost(&sg.base, sg.cap) != cudaSuccess) {
        sg.base = nullptr;
        sg.cap = 0;
        ok = false;
      }
    }
    std::string err;
    sg.used = 0;
    P->vox_cap = slot_voxel_capacity(*r.host);
    ok = ok && build_slot(*r.host, 0, r.seed, P->mem, sg, P->vox_cap, P->vox_total, P->Y, P->C, err, r.start.get()) == 0;
    ok = ok && cudaEventCreateWithFlags(&P->done, cudaEventDisableTiming) == cudaSuccess &&
         cudaEventRecord(P->done, w.st) == cudaSuccess;
    w.stage_busy[k] = cudaEventRecord(w.stage_done[k], w.st) == cudaSuccess;
    if (!ok) {
      // nothing enqueued may write the word or read the memory once the stream has drained
      P->mem.release();
      cudaStreamSynchronize(w.st);
      if (P->done) cudaEventDestroy(P->done);
    }
    std::lock_guard<std::mutex> lk(mu);
    prebuilt_bytes -= r.bytes_estimate;
    building--;
    if (ok) {
      P->C.budget = r.moves;
      prebuilt_bytes += P->mem.bytes;
      r.pre = std::move(P);
    } else {
      prebuilt_count--;
      free_words.push_back(word);
    }
  }

  // Worker threads: host preparation of queued requests, in submission order, and their device
  // slots built ahead on the worker's stream.
  void worker(int wi) {
    cudaSetDevice(device);
    for (;;) {
      Request* r = nullptr;
      {
        std::unique_lock<std::mutex> lk(mu);
        cv.wait(lk, [this] { return stopping || !prep_queue.empty(); });
        if (stopping) return;
        r = reqs[prep_queue.front()].get();
        prep_queue.pop_front();
      }
      prepare(*r, &wres[wi]);
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
      done_log.push_back(id);
      if (r.prepared.load(std::memory_order_acquire))
        drop_prebuilt(r);
      else
        cancelled_unprepared.push_back(id);  // its worker may still build a slot ahead for it
    } else if (r.state == kRunning) {
      const int i = r.slot;
      snapshot(i, r);  // the state as of the last completed launch
      r.state = kCancelled;
      done_log.push_back(id);
      auto f = std::find(fresh.begin(), fresh.end(), i);
      if (f != fresh.end()) {  // built but never launched: nothing on the device reads it
        fresh.erase(f);
        release(i);
      } else {
        // switched off on the device before the next launch; its memory is freed once the launch
        // in flight (which may still run it) has completed, or now if none is
        deactivate.push_back(i);
        if (inflight >= 0) {
          slots[i].request = -2;  // held until then
          deferred.push_back({i, inflight});
        } else {
          release(i);
        }
      }
    }
    return 0;
  }

  // Frees a request's slot built ahead (its preparation has finished; its build may still run:
  // the frees are ordered after it on its stream).
  void drop_prebuilt(Request& r) {
    std::unique_ptr<Prebuilt> P;
    {
      std::lock_guard<std::mutex> lk(mu);
      if (!r.pre) return;
      P = std::move(r.pre);
      prebuilt_bytes -= std::min(prebuilt_bytes, P->mem.bytes);
      prebuilt_count--;
    }
    P->mem.release();
    cudaEventSynchronize(P->done);  // the build no longer writes its word
    cudaEventDestroy(P->done);
    std::lock_guard<std::mutex> lk(mu);
    free_words.push_back(P->word);
  }

  // Frees slot i's memory on the stream that built it (ordered after that build) and gives the
  // slot back the admission stream, on which any later build of the slot at admission runs:
  // settle_admissions and the next launch wait for that stream only.
  void release(int i) {
    Slot& s = slots[i];
    used -= std::min(used.load(), s.mem.bytes);
    s.mem.release();
    s.mem.st = st2;
    s.mem.pool = pool;
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

  // Slot i's chain has finished and switched itself off on the device, so the launch in flight
  // does not touch its memory: its guest sites are copied to the host before the slot is freed,
  // with the control block's REVIVE fields (as Batch::write_revive takes them).
  int keep_final_state(int i, Request& r, std::string& err) {
    const ChainDev& C = h_chains[i];
    const SysConst& Y = h_sys[i];
    auto F = std::make_unique<Request::Final>();
    const int ng = Y.nspecies;
    F->xyz.resize(ng);
    std::vector<std::vector<double4>> a(ng);
    cudaError_t e = cudaSuccess;
    for (int g = 0; g < ng && e == cudaSuccess; g++) {
      const int n = C.nmol[g] * Y.sp[g].nsite;
      a[g].resize(n);
      if (n) e = cudaMemcpyAsync(a[g].data(), C.gsite + C.seg_off[g], sizeof(double4) * n, cudaMemcpyDeviceToHost, st3);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(st3);
    if (e != cudaSuccess) {
      err = std::string("final-state copy failed: ") + cudaGetErrorString(e);
      return -100 - (int)e;
    }
    F->chainstats.assign(1 + 14 * ng, 0.0);
    F->chainstats[0] = (double)C.prodcount;
    for (int g = 0; g < ng; g++) {
      for (const double4& p : a[g]) {
        F->xyz[g].push_back(p.x);
        F->xyz[g].push_back(p.y);
        F->xyz[g].push_back(p.z);
      }
      for (int k = 0; k < 6; k++) F->chainstats[1 + 14 * g + k] = C.stats[g][k];
      F->energy.push_back(C.energy[g]);
    }
    F->production = C.production != 0;
    F->last_dE = C.last_dE;
    r.fin = std::move(F);
    return 0;
  }

  int set_keep_final(bool on) {
    if (on && !st3 && cudaStreamCreateWithFlags(&st3, cudaStreamNonBlocking) != cudaSuccess) return -100;
    keep_final = on;
    return 0;
  }

  // REVIVE + REVCON of a finished request whose final state was kept (the deck is read again
  // for the framework and the formats).
  int write_revive(int id, const std::string& outdir, std::string& err) {
    if (id < 0 || id >= nreqs()) {
      err = "bad request id";
      return -1;
    }
    Request& r = req(id);
    if (r.state != kDone || !r.fin) {
      err = "the request has not finished, or finished while its final state was not kept";
      return -1;
    }
    InputDeck d;
    int rc = read_input_deck(r.dir, d, err);
    if (rc) return rc;
    if ((int)r.fin->xyz.size() != (int)d.guests.size()) {
      err = "the request's deck changed since it ran";
      return -2;
    }
    Revive rv = revive_state(d, r.fin->production, r.fin->xyz, r.fin->chainstats, r.fin->energy);
    rc = fmc::write_revive(outdir + "/REVIVE", rv, err);
    if (!rc) rc = fmc::write_revcon(outdir + "/REVCON", d, rv, r.fin->last_dE, err);
    return rc;
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
    v[18] = 0.0;
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
    r.start.reset();
    for (int id = (int)reqs.size() - 1; id >= 0; id--)
      if (reqs[id].get() == &r) {
        done_log.push_back(id);
        break;
      }
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
    long long vox_cap = slot_voxel_capacity(*r.host);
    if (r.pre) {  // built ahead by a worker (its build has completed): install it
      std::unique_ptr<Prebuilt> P = std::move(r.pre);
      const long long total = *P->vox_total;
      cudaEventDestroy(P->done);
      {
        std::lock_guard<std::mutex> lk(mu);
        prebuilt_bytes -= std::min(prebuilt_bytes, P->mem.bytes);
        prebuilt_count--;
        free_words.push_back(P->word);
      }
      if (total <= P->vox_cap) {
        s.mem = std::move(P->mem);
        s.vox_cap = P->vox_cap;
        h_sys[i] = P->Y;
        h_chains[i] = P->C;
        h_chains[i].sys = i;
        r.host.reset();
        r.start.reset();
        s.request = id;
        s.fresh = false;  // its lists were checked above
        fresh.push_back(i);
        r.state = kRunning;
        r.slot = i;
        admitted++;
        admit_prebuilt++;
        return s.mem.bytes;
      }
      // the lists outgrew their estimate: built again below at their exact size
      P->mem.release();
      vox_cap = total;
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
    s.vox_cap = vox_cap;
    s.mem.st = st2;  // the admission stream, which settle_admissions and the next launch wait for
    s.mem.pool = pool;
    int rc = build_slot(*r.host, i, r.seed, s.mem, stage, s.vox_cap, &h_vox_total[i], h_sys[i], h_chains[i], err,
                        r.start.get());
    if (rc) {
      s.mem.release();
      std::memset(&h_chains[i], 0, sizeof(ChainDev));
      reject(r, rc, err);
      return 0;
    }
    h_chains[i].budget = r.moves;
    s.request = id;
    s.fresh = true;
    fresh.push_back(i);
    r.state = kRunning;
    r.slot = i;
    admitted++;
    admit_built++;
    return s.mem.bytes;
  }

  // Admission: FIFO, while a slot is free, the front request is prepared and the memory budget
  // holds.  With nothing running, waits for the front request's preparation.
  void admit_queued(int running) {
    const double t0 = now_ms();
    bool dropped = false;
    for (int i = 0; i < nslots && !queue.empty(); i++) {
      if (slots[i].request != -1) continue;  // running, or cancelled with its memory still held
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
      if (r.pre) {  // its slot was built ahead: installed once that build has completed
        cudaError_t q = cudaEventQuery(r.pre->done);
        if (q == cudaErrorNotReady) {
          if (running) break;
          const double w0 = now_ms();
          q = cudaEventSynchronize(r.pre->done);
          wait_ms += now_ms() - w0;
        }
        if (q != cudaSuccess) drop_prebuilt(r);  // built again at admission, which reports the error
      }
      size_t ahead;
      {
        std::lock_guard<std::mutex> lk(mu);
        ahead = prebuilt_bytes;
      }
      if (!r.prep_rc && !r.pre && used.load() + ahead + r.bytes_estimate > budget) {
        if (r.bytes_estimate > budget) {
          queue.pop_front();
          reject(r, -10, "the request's device footprint exceeds the server's memory budget");
          i--;
          continue;
        }
        if (ahead > 0 && !dropped) {
          // the budget is held by slots built ahead for requests behind this one: free them
          // (they are built again when their turn comes) rather than wait on them; with nothing
          // running, first let the builds in progress finish so that they can be freed too
          if (!running) {
            const double w0 = now_ms();
            for (;;) {
              {
                std::lock_guard<std::mutex> lk(mu);
                if (building == 0) break;
              }
              std::this_thread::sleep_for(std::chrono::microseconds(200));
            }
            wait_ms += now_ms() - w0;
          }
          for (int q : queue)
            if (q != id) drop_prebuilt(req(q));
          dropped = true;
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
        used -= std::min(used.load(), s.mem.bytes);
        s.mem.release();
        s.vox_cap = h_vox_total[i];
        std::string e2;
        int rc = build_slot(*r.host, i, r.seed, s.mem, stage, s.vox_cap, &h_vox_total[i], h_sys[i], h_chains[i], e2,
                            r.start.get());
        if (rc == 0 && cudaStreamSynchronize(st2) != cudaSuccess) rc = -100;
        stage.used = 0;
        if (rc || (long long)h_vox_total[i] > s.vox_cap) {
          s.mem.release();
          s.request = -1;
          std::memset(&h_chains[i], 0, sizeof(ChainDev));
          fresh.erase(std::remove(fresh.begin(), fresh.end(), i), fresh.end());
          reject(r, rc ? rc : -12, rc ? e2 : "voxel lists changed size between builds");
          continue;
        }
        h_chains[i].budget = r.moves;
        used += s.mem.bytes;
      }
      r.host.reset();
      r.start.reset();
    }
    return 0;
  }

  // Completes launch buffer b: the control blocks it left, retirements, the deferred frees.
  int complete(int b, int* n_active, float* ms, std::string& err) {
    cudaError_t e = cudaEventSynchronize(ev_done[b]);
    float t = 0.f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&t, ev_start[b], ev_end[b]);
    if (e != cudaSuccess) {
      err = std::string("serving launch failed: ") + cudaGetErrorString(e);
      return -100 - (int)e;
    }
    launches++;
    launch_ms += t;
    last_moves = 0;
    int ran = 0;
    for (int i = 0; i < nslots; i++) {
      if (launched[b][i] < 0) continue;
      ran++;
      const int id = slots[i].request;
      // cancelled while this launch ran, or retired by the launch before and taken by a new request
      if (id != launched[b][i]) continue;
      last_moves += h_out[b][i].moves_done - h_chains[i].moves_done;
      h_chains[i] = h_out[b][i];
      const ChainDev& C = h_chains[i];
      if ((C.budget > 0 && C.moves_done >= C.budget) || !C.lgchk || C.status) {
        // the chain switched itself off on the device: the launch queued behind this one skips it
        Request& r = req(id);
        snapshot(i, r);
        if (keep_final && !C.status) {
          int rc = keep_final_state(i, r, err);
          if (rc) return rc;
        }
        r.state = C.status ? kRejected : kDone;
        if (C.status) r.err = C.status == 75 ? "too many atoms in specified system" : "chain stopped with an unknown status";
        done_log.push_back(id);
        release(i);
        retired++;
      }
    }
    moves_run += last_moves;
    for (size_t k = 0; k < deferred.size();) {
      if (deferred[k].second == b) {
        release(deferred[k].first);
        deferred.erase(deferred.begin() + k);
      } else {
        k++;
      }
    }
    if (n_active) *n_active = ran;
    if (ms) *ms = t;
    return 0;
  }

  // Queues one launch of every running slot into buffer b, after the uploads of the slots admitted
  // or cancelled since the last launch; the control blocks come back to h_out[b].
  int enqueue_launch(int moves, int b, std::string& err) {
    cudaError_t e = cudaSuccess;
    // cancelled slots first: a slot cancelled and then taken by a new request gets the new block
    for (int i : deactivate)
      if (e == cudaSuccess) e = cudaMemcpyAsync(&d_chains[i].active, h_zero, sizeof(int), cudaMemcpyHostToDevice, st);
    if (!fresh.empty() && e == cudaSuccess) e = cudaStreamWaitEvent(st, ev_admit, 0);  // their set-up
    for (int i : fresh) {
      if (e == cudaSuccess) e = cudaMemcpyAsync(d_sys + i, h_sys + i, sizeof(SysConst), cudaMemcpyHostToDevice, st);
      if (e == cudaSuccess)
        e = cudaMemcpyAsync(d_chains + i, h_chains + i, sizeof(ChainDev), cudaMemcpyHostToDevice, st);
      slots[i].fresh = false;
    }
    fresh.clear();
    deactivate.clear();
    for (int i = 0; i < nslots; i++) launched[b][i] = slots[i].request >= 0 ? slots[i].request : -1;
    BatchLaunch L;
    std::memset(&L, 0, sizeof(L));
    L.chains = d_chains;
    L.systems = d_sys;
    L.nchains = nslots;
    L.moves = moves;
    L.kmax_smem = kcap;
    L.retire_finished = 1;
    if (e == cudaSuccess) e = cudaEventRecord(ev_start[b], st);
    if (e == cudaSuccess) e = launch_batch(L, smem, tab_stride, st);
    if (e == cudaSuccess) e = cudaEventRecord(ev_end[b], st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(h_out[b], d_chains, sizeof(ChainDev) * nslots, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaEventRecord(ev_done[b], st);
    if (e != cudaSuccess) {
      err = std::string("serving launch failed: ") + cudaGetErrorString(e);
      return -100 - (int)e;
    }
    return 0;
  }

  int running_slots() const {
    int n = 0;
    for (const Slot& sl : slots) n += sl.request >= 0;
    return n;
  }

  // One step: queue the next launch, then complete the one before it (see the file comment).
  int step(int moves, int* n_active, int* n_queued, float* ms, std::string& err) {
    cudaSetDevice(device);
    if (n_active) *n_active = 0;
    if (ms) *ms = 0.f;
    int rc = 0;
    // requests cancelled during their preparation: the slots their workers built ahead are freed
    for (size_t k = 0; k < cancelled_unprepared.size();) {
      Request& r = req(cancelled_unprepared[k]);
      if (!r.prepared.load(std::memory_order_acquire)) {
        k++;
        continue;
      }
      drop_prebuilt(r);
      r.host.reset();
      r.start.reset();
      cancelled_unprepared.erase(cancelled_unprepared.begin() + k);
    }
    if (!fresh.empty()) {  // last step's admissions: set up and checked before their first launch
      rc = settle_admissions(err);
      if (rc) return rc;
    }
    if (inflight < 0 && running_slots() == 0 && !queue.empty()) {  // idle device: admit first
      admit_queued(0);
      rc = settle_admissions(err);
      if (rc) return rc;
    }
    const int prev = inflight;
    inflight = -1;
    if (running_slots() > 0) {
      const int b = next_buf;
      next_buf ^= 1;
      rc = enqueue_launch(moves, b, err);
      if (rc) return rc;
      inflight = b;
    }
    if (prev >= 0) {
      rc = complete(prev, n_active, ms, err);
      if (rc) return rc;
    }
    if (inflight >= 0 || running_slots() == 0) {
      admit_queued(inflight >= 0);  // built beside the launch in flight, launched by the next step
      if (!fresh.empty()) cudaEventRecord(ev_admit, st2);
    }
    if (n_queued) *n_queued = (int)queue.size();
    return 0;
  }

  // Requests that reached a final state since the last call (at most cap of them).
  int poll_done(int* ids, int* states, double* results, int cap) {
    const int n = std::min<int>(cap, (int)done_log.size());
    for (int k = 0; k < n; k++) {
      const Request& r = req(done_log[k]);
      if (ids) ids[k] = done_log[k];
      if (states) states[k] = r.state;
      if (results) std::memcpy(results + 32 * k, r.result, sizeof(r.result));
    }
    done_log.erase(done_log.begin(), done_log.begin() + n);
    return n;
  }

  bool busy() const { return inflight >= 0 || running_slots() > 0 || !queue.empty(); }
};

}  // namespace fmc

struct fmc_server {
  fmc::Server impl;
};

extern "C" {

int fmc_deck_footprint(const char* dir, double voxel_edge, long long* bytes, double* move_cost) {
  if (!dir || !(voxel_edge >= 1.0 && voxel_edge <= 4.0)) {
    fmc::set_last_error("bad deck directory or voxel edge (1-4 A)");
    return -1;
  }
  fmc::HostSystem h;
  std::string err;
  int rc = fmc::prepare_system(dir, h, err, voxel_edge);
  if (rc) {
    fmc::set_last_error(err);
    return rc;
  }
  if (bytes) *bytes = (long long)fmc::Server::slot_bytes_estimate(h);
  if (move_cost) {
    // algorithmic bytes of one move of an empty framework: S(k), akk and S_new (40 B a k-vector)
    // and 4.5 sites' neighbours within rcut (36 B each)
    const double nrc = (double)h.nf / h.cell.volm * (4.0 / 3.0 * fmc::kPi * h.rcut * h.rcut * h.rcut);
    *move_cost = 40.0 * h.K + 4.5 * nrc * 36.0;
  }
  return 0;
}

int fmc_server_set_voxel_edge(fmc_server* s, double edge) {
  if (!s || !(edge >= 1.0 && edge <= 4.0)) {
    fmc::set_last_error("bad server handle or voxel edge (1-4 A)");
    return -1;
  }
  s->impl.voxel_edge.store(edge);
  return 0;
}

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

int fmc_server_keep_final_state(fmc_server* s, int enable) {
  if (!s) {
    fmc::set_last_error("bad server handle");
    return -1;
  }
  if (s->impl.set_keep_final(enable != 0)) {
    fmc::set_last_error("cannot create the final-state copy stream");
    return -100;
  }
  return 0;
}

int fmc_server_write_revive(fmc_server* s, int request_id, const char* outdir) {
  if (!s || !outdir) {
    fmc::set_last_error("bad server handle or directory");
    return -1;
  }
  std::string err;
  int rc = s->impl.write_revive(request_id, outdir, err);
  if (rc) fmc::set_last_error(err);
  return rc;
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

int fmc_server_poll_done(fmc_server* s, int* ids, int* states, double* results, int cap, int* n) {
  if (!s || cap < 0 || !n) {
    fmc::set_last_error("bad server handle or capacity");
    return -1;
  }
  *n = s->impl.poll_done(ids, states, results, cap);
  return 0;
}

int fmc_server_busy(fmc_server* s, int* busy) {
  if (!s || !busy) {
    fmc::set_last_error("bad server handle");
    return -1;
  }
  *busy = s->impl.busy() ? 1 : 0;
  return 0;
}

int fmc_server_memory(fmc_server* s, long long* used, long long* budget) {
  if (!s) {
    fmc::set_last_error("bad server handle");
    return -1;
  }
  if (used) *used = (long long)s->impl.used.load();
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
  out[10] = (double)v.prep_host_us.load() / 1000.0;
  out[11] = (double)v.prep_dev_us.load() / 1000.0;
  out[12] = (double)v.admit_prebuilt;
  out[13] = (double)v.admit_built;
  return 0;
}

}  // extern "C"
