// Serving slots: the device side of admitting one request, stream-ordered on the server's
// stream with allocations from its memory pool.  The slot holds only what the batched kernel
// reads: framework atoms, inlined voxel lists, erfc / vdW tables (FP64 and FP32), the k-vector
// tables, the framework S(k) (ewald1 over the framework, ewald.f:368-630) and the chain's S(k)
// and guest segments.
#include <algorithm>
#include <cstring>

#include "fmc_batch.h"

namespace fmc {

cudaError_t SlotMemory::alloc(void** p, size_t n) {
  n = std::max<size_t>(n, 16);
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
}

namespace {

template <class T>
cudaError_t put(SlotMemory& m, const T** out, const T* src, size_t n) {
  T* p = nullptr;
  cudaError_t e = m.alloc((void**)&p, n * sizeof(T));
  if (e == cudaSuccess && n) e = cudaMemcpyAsync(p, src, n * sizeof(T), cudaMemcpyHostToDevice, m.st);
  *out = p;
  return e;
}

template <class T>
cudaError_t put(SlotMemory& m, const T** out, const std::vector<T>& v) {
  return put(m, out, v.data(), v.size());
}

}  // namespace

int build_slot(const HostSystem& h, int slot, const int seed[4], SlotMemory& mem, SysConst& Y, ChainDev& C,
               std::string& err) {
  DevSystem v;
  std::memset(&v, 0, sizeof(v));
  v.cell = h.cell;
  v.nf = h.nf;
  cudaStream_t st = mem.st;
  cudaError_t e;
  std::vector<double4> fw(h.nf);
  for (int i = 0; i < h.nf; i++) fw[i] = make_double4(h.fx[i], h.fy[i], h.fz[i], h.fq[i]);
  std::vector<float> ef(h.erc.begin(), h.erc.end()), vf(h.vvv.begin(), h.vvv.end());
  std::vector<int> kp(h.K);
  for (int k = 0; k < h.K; k++) kp[k] = kpack(h.kl[k], h.km[k], h.kn[k]);
  const int nv = h.nvox[0] * h.nvox[1] * h.nvox[2];
  std::vector<int> cnt(nv), offv(nv + 1, 0);
  int* counts = nullptr;
  double2* skfw = nullptr;
  double* scratch = nullptr;
  double* parts = nullptr;
  if ((e = put(mem, &v.fw, fw)) != cudaSuccess) goto fail;
  if ((e = put(mem, &v.fw_type, h.ftype)) != cudaSuccess) goto fail;
  for (int a = 0; a < 3; a++) v.nvox[a] = h.nvox[a];
  // voxel lists: count per voxel on the device, prefix on the host (one wait), ordered fill
  if ((e = cudaMallocFromPoolAsync((void**)&counts, sizeof(int) * nv, mem.pool, st)) != cudaSuccess) goto fail;
  e = launch_voxel_count(h.cell, h.nvox, v.fw, h.nf, h.vox_lim2, counts, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(cnt.data(), counts, sizeof(int) * nv, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  cudaFreeAsync(counts, st);
  if (e != cudaSuccess) goto fail;
  for (int i = 0; i < nv; i++) offv[i + 1] = offv[i] + cnt[i];
  {
    const size_t ne = (size_t)offv[nv];
    double4* xyzq = nullptr;
    unsigned char* vt = nullptr;
    if ((e = put(mem, &v.vox_off, offv)) != cudaSuccess) goto fail;
    if ((e = mem.alloc((void**)&xyzq, sizeof(double4) * ne)) != cudaSuccess) goto fail;
    if ((e = mem.alloc((void**)&vt, ne)) != cudaSuccess) goto fail;
    e = launch_voxel_fill(h.cell, h.nvox, v.fw, v.fw_type, h.nf, h.vox_lim2, v.vox_off, nullptr, nullptr, xyzq, vt, st);
    if (e != cudaSuccess) goto fail;
    v.vox_xyzq = xyzq;
    v.vox_type = vt;
  }
  v.rcut2 = h.rcut * h.rcut;
  v.rdr_e = 1.0 / h.drewd;
  v.rdr_v = 1.0 / h.dlrpot;
  if ((e = put(mem, &v.erc, h.erc)) != cudaSuccess) goto fail;
  if ((e = put(mem, &v.vvv, h.vvv)) != cudaSuccess) goto fail;
  if ((e = put(mem, &v.erc_f, ef)) != cudaSuccess) goto fail;
  if ((e = put(mem, &v.vvv_f, vf)) != cudaSuccess) goto fail;
  v.tab_stride = h.mxgrid + 1;
  v.ntypes = h.ntypes;
  if ((e = put(mem, &v.pair_row, h.pair_row)) != cudaSuccess) goto fail;
  v.K = h.K;
  for (int a = 0; a < 3; a++) v.kmax[a] = h.deck.kmax[a];
  if ((e = put(mem, &v.kpack, kp)) != cudaSuccess) goto fail;
  if ((e = put(mem, &v.akk, h.akk)) != cudaSuccess) goto fail;
  v.recip_pref = h.recip_pref;
  // framework S(k); the scratch goes back to the pool once the kernels have run
  if ((e = mem.alloc((void**)&skfw, sizeof(double2) * std::max(h.K, 1))) != cudaSuccess) goto fail;
  e = cudaMallocFromPoolAsync((void**)&scratch, sizeof(double) * std::max<size_t>(recip_scratch_doubles(v, h.nf), 1),
                              mem.pool, st);
  if (e == cudaSuccess)
    e = cudaMallocFromPoolAsync((void**)&parts, sizeof(double) * (recip_nparts(v) + 1), mem.pool, st);
  if (e == cudaSuccess) e = launch_recip_full(v, v.fw, h.nf, skfw, scratch, parts, st);
  if (scratch) cudaFreeAsync(scratch, st);
  if (parts) cudaFreeAsync(parts, st);
  if (e != cudaSuccess) goto fail;
  {
    int ts = 0;
    int rc = fill_sysconst(h, v, Y, &ts, err);
    if (rc) return rc;
    Y.sk_fw = skfw;
    DevAllocFn alloc = [&mem](void** p, size_t n) { return mem.alloc(p, n); };
    // an empty framework: guest energy 0 (single_point, gcmc.f:2518-2710)
    return init_chain_state(h.deck, h, skfw, 0.0, slot, seed, C, alloc, st, err);
  }
fail:
  err = std::string("slot set-up failed on the device: ") + cudaGetErrorString(e);
  return -100 - (int)e;
}

}  // namespace fmc
