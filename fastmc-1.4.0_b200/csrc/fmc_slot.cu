// Serving slots: the device side of admitting one request, enqueued on the admission stream with
// allocations from the server's memory pool and every host array staged into pinned memory, so
// admitting needs no wait.  The slot holds only what the batched kernel reads: framework atoms,
// inlined voxel lists, erfc / vdW tables, the k-vector tables, the framework S(k)
// (ewald1 over the framework, ewald.f:368-630) and the chain's S(k) and guest segments.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "fmc_batch.h"

namespace fmc {

cudaError_t SlotMemory::reserve(size_t n) {
  void* p = nullptr;
  n = (n + 255) & ~size_t(255);
  cudaError_t e = pool ? cudaMallocFromPoolAsync(&p, n, pool, st) : cudaMallocAsync(&p, n, st);
  if (e == cudaSuccess) {
    ptrs.push_back(p);
    bytes += n;
    arena = (unsigned char*)p;
    arena_cap = n;
    arena_used = 0;
  }
  return e;
}

cudaError_t SlotMemory::alloc(void** p, size_t n) {
  n = std::max<size_t>(n, 16);
  const size_t need = (n + 255) & ~size_t(255);
  if (arena && arena_used + need <= arena_cap) {
    *p = arena + arena_used;
    arena_used += need;
    return cudaSuccess;
  }
  cudaError_t e = pool ? cudaMallocFromPoolAsync(p, n, pool, st) : cudaMallocAsync(p, n, st);
  if (e == cudaSuccess) {
    ptrs.push_back(*p);
    bytes += n;
  }
  return e;
}

void SlotMemory::release() {
  for (void* p : ptrs) cudaFreeAsync(p, st);
  ptrs.clear();
  bytes = 0;
  arena = nullptr;
  arena_cap = arena_used = 0;
}

void* Staging::take(size_t n) {
  size_t at = (used + 255) & ~size_t(255);
  if (at + n > cap) return nullptr;
  used = at + n;
  return base + at;
}

namespace {

size_t al(size_t n) { return (n + 255) & ~size_t(255); }

// Host arrays of a system in the order they are staged, with their byte sizes.
struct Parts {
  size_t fw, ftype, erc, vvv, prow, kp, akk;
  explicit Parts(const HostSystem& h)
      : fw(sizeof(double4) * h.nf),
        ftype(sizeof(int) * h.nf),
        erc(sizeof(double) * h.erc.size()),
        vvv(sizeof(double) * h.vvv.size()),
        prow(sizeof(int) * h.pair_row.size()),
        kp(sizeof(int) * h.K),
        akk(sizeof(double) * h.K) {}
  size_t total() const {
    return al(fw) + al(ftype) + al(erc) + al(vvv) + al(prow) + al(kp) + al(akk);
  }
};

// The guests a slot starts with, over the chain state init_chain_state enqueued (framework
// S(k), no guests): S(k) of every atom and the sites, copied from pageable host memory in stream
// order (each copy has read its source when it returns), and the control block's counts.  The
// counts follow the batched path's preloaded guests (init_chain) and REVIVE restart
// (Batch::restart, gcmc.f:396-409, 547-556).
int load_slot_start(const HostSystem& h, const SlotStart& s, ChainDev& C, cudaStream_t st, std::string& err) {
  const InputDeck& d = h.deck;
  const int ng = (int)d.guests.size();
  if ((int)s.sk.size() != h.K || (int)s.nmol.size() != ng || (int)s.sites.size() != ng || (int)s.types.size() != ng ||
      (s.from_revive && (int)s.chainstats.size() != 1 + 14 * ng)) {
    err = "slot start state does not match the deck";
    return -12;
  }
  for (int g = 0; g < ng; g++)
    if (s.nmol[g] * d.guests[g].nsite > C.seg_cap[g] || (int)s.sites[g].size() != s.nmol[g] * d.guests[g].nsite ||
        s.types[g].size() != s.sites[g].size()) {
      err = "guests of the start state exceed the chain's capacity (max guest atoms)";
      return -75;
    }
  cudaError_t e = h.K ? cudaMemcpyAsync(C.sk, s.sk.data(), sizeof(double2) * h.K, cudaMemcpyHostToDevice, st)
                      : cudaSuccess;
  for (int g = 0; g < ng && e == cudaSuccess; g++) {
    const size_t n = s.sites[g].size();
    if (!n) continue;
    e = cudaMemcpyAsync(C.gsite + C.seg_off[g], s.sites[g].data(), sizeof(double4) * n, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(C.gtype + C.seg_off[g], s.types[g].data(), sizeof(int) * n, cudaMemcpyHostToDevice, st);
  }
  if (e != cudaSuccess) {
    err = std::string("slot start upload failed: ") + cudaGetErrorString(e);
    return -100 - (int)e;
  }
  for (int g = 0; g < ng; g++) {
    C.nmol[g] = s.nmol[g];
    C.totatm += (int)s.sites[g].size();
    for (int t : s.types[g]) C.numtyp[t]++;
  }
  if (s.from_revive) {
    for (int g = 0; g < ng; g++)
      for (int k = 0; k < 6; k++) C.stats[g][k] = s.chainstats[1 + 14 * g + k];
    C.prodcount = 0;
    C.last_dE = 0.0;
    C.production = s.production;
    if (C.production && C.eqsteps > 0) C.production = 0;  // gcmc.f:396-409
    if (C.eqsteps == 0) C.production = 1;                 // gcmc.f:553-554
  }
  return 0;
}

}  // namespace

size_t slot_staging_bytes(const HostSystem& h) { return Parts(h).total() + 256; }

long long slot_voxel_capacity(const HostSystem& h) {
  // every atom appears in the lists of the voxels whose centres lie within lim of it
  const double lim = std::sqrt(h.vox_lim2);
  const double nv = (double)h.nvox[0] * h.nvox[1] * h.nvox[2];
  const double per_atom = std::min(nv, 4.0 / 3.0 * kPi * lim * lim * lim / (h.cell.volm / nv));
  return (long long)(1.15 * h.nf * per_atom) + 4096;
}

int build_slot(const HostSystem& h, int slot, const int seed[4], SlotMemory& mem, Staging& stg, long long vox_cap,
               int* vox_total, SysConst& Y, ChainDev& C, std::string& err, const SlotStart* start) {
  DevSystem v;
  std::memset(&v, 0, sizeof(v));
  v.cell = h.cell;
  v.nf = h.nf;
  cudaStream_t st = mem.st;
  cudaError_t e = cudaSuccess;
  const Parts P(h);
  const size_t total = P.total();
  unsigned char* hs = (unsigned char*)stg.take(total);
  if (!hs) {
    err = "slot staging buffer full";
    return -11;
  }
  // stage every host array, then one copy into one device block with the same layout
  size_t o = 0;
  auto place = [&](size_t n) {
    size_t at = o;
    o += al(n);
    return at;
  };
  const size_t o_fw = place(P.fw), o_ft = place(P.ftype), o_erc = place(P.erc), o_vvv = place(P.vvv),
               o_prow = place(P.prow), o_kp = place(P.kp),
               o_akk = place(P.akk);
  {
    double4* fw = (double4*)(hs + o_fw);
    for (int i = 0; i < h.nf; i++) fw[i] = make_double4(h.fx[i], h.fy[i], h.fz[i], h.fq[i]);
    std::memcpy(hs + o_ft, h.ftype.data(), P.ftype);
    std::memcpy(hs + o_erc, h.erc.data(), P.erc);
    std::memcpy(hs + o_vvv, h.vvv.data(), P.vvv);
    std::memcpy(hs + o_prow, h.pair_row.data(), P.prow);
    int* kp = (int*)(hs + o_kp);
    for (int k = 0; k < h.K; k++) kp[k] = kpack(h.kl[k], h.km[k], h.kn[k]);
    std::memcpy(hs + o_akk, h.akk.data(), P.akk);
  }
  unsigned char* d = nullptr;
  const int nv = h.nvox[0] * h.nvox[1] * h.nvox[2];
  if (vox_cap <= 0) vox_cap = slot_voxel_capacity(h);
  const bool prefilter = voxel_prefilter_applies(h.cell, h.nvox) && h.nf > 0;
  v.K = h.K;
  for (int a = 0; a < 3; a++) v.kmax[a] = h.deck.kmax[a];
  int* counts = nullptr;
  unsigned* code = nullptr;
  int* off = nullptr;
  double4* xyzq = nullptr;
  unsigned char* vt = nullptr;
  double2* skfw = nullptr;
  double* scratch = nullptr;
  double* parts = nullptr;
  {
    // every buffer of the slot, set-up scratch included, from one pool allocation
    const size_t arena = total + al(sizeof(int) * nv) + (prefilter ? al(sizeof(unsigned) * h.nf) : 0) +
                         al(sizeof(int) * (nv + 1)) + al(sizeof(double4) * vox_cap) + al(vox_cap) +
                         al(sizeof(double2) * std::max(h.K, 1)) +
                         al(sizeof(double) * std::max<size_t>(recip_scratch_doubles(v, h.nf), 1)) +
                         al(sizeof(double) * (recip_nparts(v) + 1)) + chain_state_bytes(h.deck, h, true) + 16 * 256;
    if ((e = mem.reserve(arena)) != cudaSuccess) goto fail;
  }
  if ((e = mem.alloc((void**)&d, total)) != cudaSuccess) goto fail;
  if ((e = cudaMemcpyAsync(d, hs, total, cudaMemcpyHostToDevice, st)) != cudaSuccess) goto fail;
  v.fw = (const double4*)(d + o_fw);
  v.fw_type = (const int*)(d + o_ft);
  v.erc = (const double*)(d + o_erc);
  v.vvv = (const double*)(d + o_vvv);
  v.pair_row = (const int*)(d + o_prow);
  v.kpack = (const int*)(d + o_kp);
  v.akk = (const double*)(d + o_akk);
  for (int a = 0; a < 3; a++) v.nvox[a] = h.nvox[a];
  // voxel lists: count, device prefix sum, fill up to the capacity
  if ((e = mem.alloc((void**)&counts, sizeof(int) * nv)) != cudaSuccess) goto fail;
  if ((e = mem.alloc((void**)&off, sizeof(int) * (nv + 1))) != cudaSuccess) goto fail;
  if ((e = mem.alloc((void**)&xyzq, sizeof(double4) * vox_cap)) != cudaSuccess) goto fail;
  if ((e = mem.alloc((void**)&vt, vox_cap)) != cudaSuccess) goto fail;
  if (prefilter) {
    if ((e = mem.alloc((void**)&code, sizeof(unsigned) * h.nf)) != cudaSuccess) goto fail;
    e = launch_voxel_codes(h.cell, h.nvox, v.fw, h.nf, code, st);
  }
  if (e == cudaSuccess) e = launch_voxel_count(h.cell, h.nvox, v.fw, h.nf, h.vox_lim2, code, counts, st);
  if (e == cudaSuccess) e = launch_exclusive_scan(counts, nv, off, st);
  if (e == cudaSuccess)
    e = launch_voxel_fill(h.cell, h.nvox, v.fw, v.fw_type, h.nf, h.vox_lim2, code, off, nullptr, nullptr, xyzq, vt,
                          vox_cap, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(vox_total, off + nv, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (e != cudaSuccess) goto fail;
  v.vox_off = off;
  v.vox_xyzq = xyzq;
  v.vox_type = vt;
  v.rcut2 = h.rcut * h.rcut;
  v.rdr_e = 1.0 / h.drewd;
  v.rdr_v = 1.0 / h.dlrpot;
  v.tab_stride = h.mxgrid + 1;
  v.ntypes = h.ntypes;
  v.recip_pref = h.recip_pref;
  // framework S(k)
  if ((e = mem.alloc((void**)&skfw, sizeof(double2) * std::max(h.K, 1))) != cudaSuccess) goto fail;
  e = mem.alloc((void**)&scratch, sizeof(double) * std::max<size_t>(recip_scratch_doubles(v, h.nf), 1));
  if (e == cudaSuccess) e = mem.alloc((void**)&parts, sizeof(double) * (recip_nparts(v) + 1));
  if (e == cudaSuccess) e = launch_recip_full(v, v.fw, h.nf, skfw, scratch, parts, st);
  if (e != cudaSuccess) goto fail;
  {
    int ts = 0;
    int rc = fill_sysconst(h, v, Y, &ts, err);
    if (rc) return rc;
    DevAllocFn alloc = [&mem](void** p, size_t n) { return mem.alloc(p, n); };
    // an empty framework: guest energy 0 (single_point, gcmc.f:2518-2710)
    if (!start) return init_chain_state(h.deck, h, skfw, 0.0, slot, seed, C, alloc, st, err, true);
    rc = init_chain_state(h.deck, h, skfw, start->spenergy, slot, seed, C, alloc, st, err, true);
    if (rc) return rc;
    return load_slot_start(h, *start, C, st, err);
  }
fail:
  err = std::string("slot set-up failed on the device: ") + cudaGetErrorString(e);
  return -100 - (int)e;
}

}  // namespace fmc
