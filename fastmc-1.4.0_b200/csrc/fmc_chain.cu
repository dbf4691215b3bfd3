// Chain: device upload, single-point set-up and the plain-path host move loop.
#include <atomic>
#include "fmc_chain.h"
#include "fmc_restart.h"

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstring>

namespace fmc {

#define FMC_CUDA(expr)                         \
  do {                                         \
    cudaError_t e_ = (expr);                   \
    if (e_ != cudaSuccess) return sync_error(e_, &err); \
  } while (0)

namespace {

template <class T>
cudaError_t dalloc(std::vector<void*>& keep, T** p, size_t n) {
  cudaError_t e = cudaMalloc((void**)p, std::max<size_t>(n, 1) * sizeof(T));
  if (e == cudaSuccess) keep.push_back(*p);
  return e;
}

template <class T>
cudaError_t upload(std::vector<void*>& keep, const T** out, const std::vector<T>& v) {
  T* p = nullptr;
  cudaError_t e = dalloc(keep, &p, v.size());
  if (e != cudaSuccess) return e;
  if (!v.empty()) e = cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice);
  *out = p;
  return e;
}

}  // namespace

DeviceSystem::~DeviceSystem() {
  int cur = 0;
  cudaGetDevice(&cur);
  cudaSetDevice(device);
  for (void* p : allocations) cudaFree(p);
  cudaSetDevice(cur);
}

int upload_system(const HostSystem& h, DeviceSystem& d, std::string& err) {
  DevSystem& v = d.view;
  v.cell = h.cell;
  v.nf = h.nf;
  std::vector<double4> fw(h.nf);
  for (int i = 0; i < h.nf; i++) fw[i] = make_double4(h.fx[i], h.fy[i], h.fz[i], h.fq[i]);
  cudaError_t e;
  if ((e = upload(d.allocations, &v.fw, fw)) != cudaSuccess) goto fail;
  if ((e = upload(d.allocations, &v.fw_type, h.ftype)) != cudaSuccess) goto fail;
  for (int a = 0; a < 3; a++) v.nvox[a] = h.nvox[a];
  {
    // voxel lists built on the device: count per voxel, prefix sum, ordered fill
    const int nv = h.nvox[0] * h.nvox[1] * h.nvox[2];
    int* counts = nullptr;
    unsigned* code = nullptr;  // per-atom voxel codes of an orthorhombic cell (list prefilter)
    if ((e = cudaMalloc(&counts, sizeof(int) * nv)) != cudaSuccess) goto fail;
    if (voxel_prefilter_applies(h.cell, h.nvox) && h.nf > 0) {
      if ((e = cudaMalloc(&code, sizeof(unsigned) * h.nf)) != cudaSuccess) {
        cudaFree(counts);
        goto fail;
      }
      e = launch_voxel_codes(h.cell, h.nvox, v.fw, h.nf, code, 0);
    }
    if (e == cudaSuccess) e = launch_voxel_count(h.cell, h.nvox, v.fw, h.nf, h.vox_lim2, code, counts, 0);
    std::vector<int> cnt(nv), offv(nv + 1, 0);
    if (e == cudaSuccess) e = cudaMemcpy(cnt.data(), counts, sizeof(int) * nv, cudaMemcpyDeviceToHost);
    cudaFree(counts);
    if (e != cudaSuccess) {
      cudaFree(code);
      goto fail;
    }
    for (int i = 0; i < nv; i++) offv[i + 1] = offv[i] + cnt[i];
    const size_t ne = (size_t)offv[nv];
    d.vox_entries = (long long)ne;
    int* atoms = nullptr;
    unsigned short* a16 = nullptr;
    double4* xyzq = nullptr;
    unsigned char* vt = nullptr;
    e = upload(d.allocations, &v.vox_off, offv);
    if (e == cudaSuccess) e = dalloc(d.allocations, &atoms, ne);
    if (e == cudaSuccess && h.nf <= 65535) e = dalloc(d.allocations, &a16, ne);
    if (e == cudaSuccess) e = dalloc(d.allocations, &xyzq, ne);
    if (e == cudaSuccess) e = dalloc(d.allocations, &vt, ne);
    if (e == cudaSuccess)
      e = launch_voxel_fill(h.cell, h.nvox, v.fw, v.fw_type, h.nf, h.vox_lim2, code, v.vox_off, atoms, a16, xyzq, vt,
                            (long long)ne, 0);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    cudaFree(code);
    if (e != cudaSuccess) goto fail;
    v.vox_atoms = atoms;
    v.vox_atoms16 = a16;
    v.vox_xyzq = xyzq;
    v.vox_type = vt;
  }
  v.rcut2 = h.rcut * h.rcut;
  v.rdr_e = 1.0 / h.drewd;
  v.rdr_v = 1.0 / h.dlrpot;
  if ((e = upload(d.allocations, &v.erc, h.erc)) != cudaSuccess) goto fail;
  if ((e = upload(d.allocations, &v.vvv, h.vvv)) != cudaSuccess) goto fail;
  v.tab_stride = h.mxgrid + 1;
  v.ntypes = h.ntypes;
  if ((e = upload(d.allocations, &v.pair_row, h.pair_row)) != cudaSuccess) goto fail;
  v.K = h.K;
  for (int a = 0; a < 3; a++) v.kmax[a] = h.deck.kmax[a];
  {
    std::vector<int> kp(h.K);
    for (int k = 0; k < h.K; k++) kp[k] = kpack(h.kl[k], h.km[k], h.kn[k]);
    if ((e = upload(d.allocations, &v.kpack, kp)) != cudaSuccess) goto fail;
  }
  if ((e = upload(d.allocations, &v.akk, h.akk)) != cudaSuccess) goto fail;
  v.recip_pref = h.recip_pref;
  return 0;
fail:
  err = std::string("device upload failed: ") + cudaGetErrorString(e);
  return -1;
}

void Chain::close_outputs() {
  for (std::FILE* f : numg_f)
    if (f) std::fclose(f);
  for (std::FILE* f : his_f)
    if (f) std::fclose(f);
  numg_f.clear();
  his_f.clear();
}

int Chain::open_outputs(const std::string& dir, std::string& err) {
  close_outputs();
  if (dir.empty()) return 0;
  const int ng = (int)sp.size();
  for (int i = 0; i < ng; i++) {
    char a[64], b[64];
    if (ng > 1) {
      std::snprintf(a, sizeof(a), "/numguests%02d.out", i + 1);
      std::snprintf(b, sizeof(b), "/his%02d.xyz", i + 1);
    } else {
      std::snprintf(a, sizeof(a), "/numguests.out");
      std::snprintf(b, sizeof(b), "/his.xyz");
    }
    numg_f.push_back(std::fopen((dir + a).c_str(), "w"));
    if (sys.deck.nhis != 0) his_f.push_back(std::fopen((dir + b).c_str(), "w"));
  }
  for (std::FILE* f : numg_f)
    if (!f) err = "cannot write numguests.out under " + dir;
  for (std::FILE* f : his_f)
    if (!f) err = "cannot write his.xyz under " + dir;
  if (!err.empty()) {
    close_outputs();
    return -1;
  }
  return 0;
}

Chain::~Chain() {
  close_outputs();
  if (ev0) cudaEventDestroy(ev0);
  if (ev1) cudaEventDestroy(ev1);
  if (st) {
    cudaSetDevice(device);
    stop_server();
    if (srv_st) cudaStreamDestroy(srv_st);
    if (mb) cudaFreeHost(mb);
    if (h_fl) cudaFreeHost(h_fl);
    if (srv_words) cudaFreeHost(srv_words);
    if (d_fl) cudaFree(d_fl);
    cudaStreamSynchronize(st);
    for (void* p : {(void*)sk, (void*)sk_new, (void*)sk_save, (void*)gsite, (void*)gtype, (void*)W.recip_part, (void*)W.site_e,
                    (void*)W.counter, (void*)recip_scratch, (void*)recip_parts, (void*)all_atoms})
      if (p) cudaFree(p);
    if (W.result) cudaFreeHost(W.result);
    cudaStreamDestroy(st);
  }
}

int Chain::sync_error(cudaError_t e, std::string* err) {
  if (err) *err = std::string("CUDA error: ") + cudaGetErrorString(e);
  return -100 - (int)e;
}

GuestView Chain::guest_view() const {
  GuestView G{};
  G.site = gsite;
  G.type = gtype;
  G.nseg = (int)sp.size();
  for (int g = 0; g < G.nseg; g++) {
    G.seg_off[g] = sp[g].seg_off;
    G.seg_len[g] = sp[g].nmol * sp[g].nsite;
  }
  return G;
}

int prepare_system(const std::string& dir, HostSystem& sys, std::string& err, double voxel_edge) {
  InputDeck deck;
  int rc = read_input_deck(dir, deck, err);
  if (rc) return rc;
  if ((int)deck.guests.size() > kMaxGuestTypes) {
    err = "more guest species than supported";
    return -5;
  }
  for (int f : deck.ffrz)
    if (f == 0) {
      err = "framework atoms must be frozen (rigid framework)";
      return -6;
    }
  return build_host_system(deck, sys, err, voxel_edge);
}

int Chain::open(const std::string& dir, const int seed[4], int dev, std::string& err, double voxel_edge) {
  HostSystem h;
  int rc = prepare_system(dir, h, err, voxel_edge);
  if (rc) return rc;
  return open_prepared(std::move(h), seed, dev, err);
}

int Chain::open_prepared(HostSystem&& prepared, const int seed[4], int dev, std::string& err) {
  sys = std::move(prepared);
  const InputDeck& deck = sys.deck;
  int rc = 0;
  device = dev;
  dsys.device = dev;
  FMC_CUDA(cudaSetDevice(dev));
  FMC_CUDA(configure_kernels());
  FMC_CUDA(configure_recip_kernels());
  FMC_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  rc = upload_system(sys, dsys, err);
  if (rc) return rc;
  const int K = sys.K, ng = (int)deck.guests.size();
  // guest segments: preloaded molecules + the reference's guest-atom budget (error 75)
  sp.assign(ng, Species());
  int off = 0;
  for (int g = 0; g < ng; g++) {
    const GuestSpecies& G = deck.guests[g];
    sp[g].nsite = G.nsite;
    sp[g].seg_off = off;
    sp[g].cap_sites = G.nmols * G.nsite + deck.maxguest;
    sp[g].nmol = G.nmols;
    sp[g].xyz = G.xyz;
    off += sp[g].cap_sites;
  }
  gcap = off;
  FMC_CUDA(cudaMalloc(&sk, sizeof(double2) * std::max(K, 1)));
  FMC_CUDA(cudaMalloc(&sk_new, sizeof(double2) * std::max(K, 1)));
  FMC_CUDA(cudaMalloc(&sk_save, sizeof(double2) * std::max(K, 1)));
  FMC_CUDA(cudaMalloc(&gsite, sizeof(double4) * std::max(gcap, 1)));
  FMC_CUDA(cudaMalloc(&gtype, sizeof(int) * std::max(gcap, 1)));
  W.gsite = gsite;
  W.gtype = gtype;
  FMC_CUDA(cudaMalloc(&W.recip_part, sizeof(double) * (pass_recip_blocks(dsys.view) + 1)));
  FMC_CUDA(cudaMalloc(&W.site_e, sizeof(double) * 2 * kMaxPassSites));
  FMC_CUDA(cudaMalloc(&W.counter, sizeof(unsigned)));
  FMC_CUDA(cudaMemset(W.counter, 0, sizeof(unsigned)));
  // the pass result goes straight to pinned host memory, which the kernel addresses through unified
  // addressing: a copy back per pass cost as much as a third of the plain path's time
  FMC_CUDA(cudaMallocHost(&W.result, sizeof(double) * 4));
  FMC_CUDA(cudaStreamCreateWithFlags(&srv_st, cudaStreamNonBlocking));
  FMC_CUDA(cudaMallocHost(&mb, sizeof(PassMailbox)));
  FMC_CUDA(cudaMallocHost(&h_fl, sizeof(PassServerFlags)));
  FMC_CUDA(cudaMallocHost(&srv_words, sizeof(int) * 2));
  FMC_CUDA(cudaMalloc(&d_fl, sizeof(PassServerFlags)));
  std::memset(mb, 0, sizeof(PassMailbox));
  srv_words[0] = srv_words[1] = 0;
  all_cap = sys.nf + gcap;
  FMC_CUDA(cudaMalloc(&all_atoms, sizeof(double4) * std::max(all_cap, 1)));
  recip_scratch_n = recip_scratch_doubles(dsys.view, all_cap);
  FMC_CUDA(cudaMalloc(&recip_scratch, sizeof(double) * recip_scratch_n));
  FMC_CUDA(cudaMalloc(&recip_parts, sizeof(double) * (recip_nparts(dsys.view) + 1)));
  // upload preloaded guests
  for (int g = 0; g < ng; g++) {
    rc = set_guests(g, sp[g].nmol, sp[g].xyz.data());
    if (rc) {
      err = "guest upload failed";
      return rc;
    }
  }
  totatm = sys.nf;
  for (auto& s : sp) totatm += s.nmol * s.nsite;
  framatm = totatm;
  rc = single_point();
  if (rc) {
    err = "single-point set-up failed on the device";
    return rc;
  }
  // move-loop state (gcmc.f:320-588)
  duni_seed(rng, seed[0], seed[1], seed[2], seed[3]);
  duni_next(rng);  // gcmc.f:335-336: the second duni() call consumes one draw
  energy.assign(ng, spenergy);
  delE.assign(ng, 0.0);
  elrc = 0.0;  // the move loop's elrc starts at zero (gcmc.f:131-132)
  delrdisp.assign(ng, deck.delr);
  tran_delr.assign(ng, deck.delr);
  accept_disp.assign(ng, 0);
  disp_count.assign(ng, 0);
  accept_tran.assign(ng, 0);
  tran_count.assign(ng, 0);
  rotangle = kPi / 3.0;
  rota_rotangle = rotangle;
  chainstats.assign(1 + 14 * ng, 0.0);
  gstpress = deck.press;
  despre = deck.despre;
  presrate = 0.0;
  std::memset(&win, 0, sizeof(win));
  gasmol.assign((size_t)ng * kSampleCap + 1, 0.0);
  gaseng.assign((size_t)ng * kSampleCap + 1, 0.0);
  prob.assign(deck.plots.size(), std::vector<double>((size_t)deck.ngrid[0] * deck.ngrid[1] * deck.ngrid[2], 0.0));
  production = (deck.eqsteps == 0);
  return 0;
}

int Chain::set_guests(int g, int nmol, const double* xyz) {
  Species& s = sp[g];
  if (nmol * s.nsite > s.cap_sites) return -75;
  if (int rc = stop_server()) return rc;
  if (int rc = flush_commit()) return rc;
  s.nmol = nmol;
  s.xyz.assign(xyz, xyz + 3 * nmol * s.nsite);
  const GuestSpecies& G = sys.deck.guests[g];
  std::vector<double4> a(std::max(nmol * s.nsite, 1));
  std::vector<int> t(std::max(nmol * s.nsite, 1));
  for (int m = 0; m < nmol; m++)
    for (int i = 0; i < s.nsite; i++) {
      int j = m * s.nsite + i;
      a[j] = make_double4(xyz[3 * j], xyz[3 * j + 1], xyz[3 * j + 2], G.charge[i]);
      t[j] = G.type[i];
    }
  cudaError_t e = cudaMemcpyAsync(gsite + s.seg_off, a.data(), sizeof(double4) * nmol * s.nsite,
                                  cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(gtype + s.seg_off, t.data(), sizeof(int) * nmol * s.nsite, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return sync_error(e);
  totatm = sys.nf;
  for (auto& x : sp) totatm += x.nmol * x.nsite;
  return 0;
}

// storeprob (utility_pack.f:496-561): every guest molecule's centre of mass and sites in
// fractional coordinates, binned into its species' plots in the reference's order.
void Chain::store_prob() {
  const InputDeck& d = sys.deck;
  const int na = d.ngrid[0], nb = d.ngrid[1], nc = d.ngrid[2];
  for (int g = 0; g < (int)sp.size(); g++) {
    const GuestSpecies& G = d.guests[g];
    const int ns = sp[g].nsite;
    for (int m = 0; m < sp[g].nmol; m++) {
      const double* x = sp[g].xyz.data() + 3 * m * ns;
      double c[3], fc[3];
      centre_of_mass(G.mass.data(), ns, x, x + 1, x + 2, 3, c);
      frac_wrap(sys.cell.rh, c[0], c[1], c[2], fc);
      for (size_t ip = 0; ip < d.plots.size(); ip++) {
        if (d.plots[ip].guest != g) continue;
        std::vector<double>& grid = prob[ip];
        auto add = [&grid](long long i, double w) { grid[i] += w; };
        for (int site : d.plots[ip].sites) {
          if (site == 0) {
            equitable_bin(na, nb, nc, fc[0], fc[1], fc[2], add);
          } else {
            double f[3];
            const double* a = x + 3 * (site - 1);
            frac_wrap(sys.cell.rh, a[0], a[1], a[2], f);
            equitable_bin(na, nb, nc, f[0], f[1], f[2], add);
          }
        }
      }
    }
  }
}

int Chain::restart(const Revive& r, std::string& err) {
  const std::vector<std::vector<double>> xyz = revive_guest_xyz(sys.deck, r);
  for (int g = 0; g < (int)sp.size(); g++) {
    const int nmol = (int)(xyz[g].size() / (3 * sp[g].nsite));
    if (set_guests(g, nmol, xyz[g].data())) {
      err = "REVIVE holds more guests than the chain's capacity (max guest atoms)";
      return -75;
    }
  }
  int rc = single_point();
  if (rc) {
    err = "single point of the restart state failed on the device";
    return rc;
  }
  energy.assign(sp.size(), spenergy);  // gcmc.f:547-556: every species starts at spenergy
  delE.assign(sp.size(), 0.0);
  if (r.chainstats.size() == chainstats.size()) chainstats = r.chainstats;
  prodcount = 0;
  production = r.production;
  if (production && sys.deck.eqsteps > 0) production = false;  // gcmc.f:396-409
  if (sys.deck.eqsteps == 0) production = true;                 // gcmc.f:553-554
  return 0;
}

// S(k) over all current atoms: guests in species order, then the framework (condense order).
int Chain::full_recip(double* e_out) {
  if (int rc0 = stop_server()) return rc0;  // nothing else runs beside the resident kernel
  if (int rc = flush_commit()) return rc;
  int n = 0;
  cudaError_t e = cudaSuccess;
  for (auto& s : sp) {
    int len = s.nmol * s.nsite;
    if (len) e = cudaMemcpyAsync(all_atoms + n, gsite + s.seg_off, sizeof(double4) * len, cudaMemcpyDeviceToDevice, st);
    n += len;
  }
  if (e == cudaSuccess && sys.nf)
    e = cudaMemcpyAsync(all_atoms + n, dsys.view.fw, sizeof(double4) * sys.nf, cudaMemcpyDeviceToDevice, st);
  n += sys.nf;
  if (e == cudaSuccess) e = launch_recip_full(dsys.view, all_atoms, n, sk, recip_scratch, recip_parts, st);
  std::vector<double> parts(recip_nparts(dsys.view));
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(parts.data(), recip_parts, sizeof(double) * parts.size(), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return sync_error(e);
  double q2 = 0.0;
  for (int g = 0; g < (int)sp.size(); g++)
    for (int m = 0; m < sp[g].nmol; m++)
      for (int i = 0; i < sp[g].nsite; i++) q2 = q2 + sys.deck.guests[g].charge[i] * sys.deck.guests[g].charge[i];
  for (int i = 0; i < sys.nf; i++) q2 = q2 + sys.fq[i] * sys.fq[i];
  double engsic = -kR4pie0 * sys.alpha * q2 / kSqrPi;
  if (e_out) *e_out = recip_energy_from_parts(dsys.view, parts.data()) + engsic;
  return 0;
}

// single_point (gcmc.f:2518-2710): framework-only and full reciprocal energies, guest
// real-space energies (guest-framework once, guest-guest halved), the intramolecular
// correction and the tail correction.
int Chain::single_point() {
  if (int rc0 = stop_server()) return rc0;  // nothing else runs beside the resident kernel
  if (int rc = flush_commit()) return rc;
  // framework only
  cudaError_t e = launch_recip_full(dsys.view, dsys.view.fw, sys.nf, sk, recip_scratch, recip_parts, st);
  std::vector<double> parts(recip_nparts(dsys.view));
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(parts.data(), recip_parts, sizeof(double) * parts.size(), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return sync_error(e);
  double q2f = 0.0;
  for (int i = 0; i < sys.nf; i++) q2f = q2f + sys.fq[i] * sys.fq[i];
  ewald1sum = recip_energy_from_parts(dsys.view, parts.data()) + (-kR4pie0 * sys.alpha * q2f / kSqrPi);
  double eall = 0.0;
  int rc = full_recip(&eall);
  if (rc) return rc;
  // numtyp / numfrz over all atoms (lrcorrect, vdw_terms.f:542-553)
  numtyp.assign(sys.ntypes + 1, 0);
  numfrz.assign(sys.ntypes + 1, 0);
  for (int i = 0; i < sys.nf; i++) {
    numtyp[sys.ftype[i]]++;
    if (sys.ffrz[i]) numfrz[sys.ftype[i]]++;
  }
  int nguest_sites = 0;
  for (int g = 0; g < (int)sp.size(); g++)
    for (int m = 0; m < sp[g].nmol; m++)
      for (int i = 0; i < sp[g].nsite; i++) {
        numtyp[sys.deck.guests[g].type[i]]++;
        nguest_sites++;
      }
  double elrc0 = lrc_energy(sys, numtyp, numfrz);
  double ewald1eng = 0, e2 = 0, ev = 0, e3 = 0;
  if (nguest_sites > 0) {
    ewald1eng = eall - ewald1sum;
    // one entry per guest site: its index and its own molecule's site range
    std::vector<int> idx, lo, hi;
    for (int g = 0; g < (int)sp.size(); g++)
      for (int m = 0; m < sp[g].nmol; m++)
        for (int i = 0; i < sp[g].nsite; i++) {
          idx.push_back(sp[g].seg_off + m * sp[g].nsite + i);
          lo.push_back(sp[g].seg_off + m * sp[g].nsite);
          hi.push_back(sp[g].seg_off + (m + 1) * sp[g].nsite);
        }
    const int n = (int)idx.size();
    int* dbuf = nullptr;
    double* dout = nullptr;
    e = cudaMalloc(&dbuf, sizeof(int) * 3 * n);
    if (e == cudaSuccess) e = cudaMalloc(&dout, sizeof(double) * 4 * n);
    std::vector<int> packed;
    packed.insert(packed.end(), idx.begin(), idx.end());
    packed.insert(packed.end(), lo.begin(), lo.end());
    packed.insert(packed.end(), hi.begin(), hi.end());
    if (e == cudaSuccess) e = cudaMemcpyAsync(dbuf, packed.data(), sizeof(int) * 3 * n, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = launch_single_point_rs(dsys.view, guest_view(), n, dbuf, dbuf + n, dbuf + 2 * n, dout, st);
    std::vector<double> out(4 * n);
    if (e == cudaSuccess) e = cudaMemcpyAsync(out.data(), dout, sizeof(double) * 4 * n, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFree(dbuf);
    cudaFree(dout);
    if (e != cudaSuccess) return sync_error(e);
    double cf = 0, vf = 0, cg = 0, vg = 0;
    for (int i = 0; i < n; i++) {
      cf += out[4 * i];
      vf += out[4 * i + 1];
      cg += out[4 * i + 2];
      vg += out[4 * i + 3];
    }
    e2 = cf + 0.5 * cg;
    ev = vf + 0.5 * vg;
    // intramolecular exclusion correction from the actual coordinates (ewald3 over the
    // exclusion lists, gcmc.f:2676-2697)
    for (int g = 0; g < (int)sp.size(); g++) {
      const GuestSpecies& G = sys.deck.guests[g];
      for (int m = 0; m < sp[g].nmol; m++) {
        const double* X = sp[g].xyz.data() + 3 * m * sp[g].nsite;
        for (int i = 0; i < sp[g].nsite; i++) {
          double part = 0.0;
          for (int j = i + 1; j < sp[g].nsite; j++) {
            double dx = X[3 * i] - X[3 * j], dy = X[3 * i + 1] - X[3 * j + 1], dz = X[3 * i + 2] - X[3 * j + 2];
            min_image(sys.cell, dx, dy, dz);
            double r = std::sqrt(dx * dx + dy * dy + dz * dz);
            part = part - ewald3_pair(sys.alpha, G.charge[i] * kR4pie0 * G.charge[j], r);
          }
          e3 = e3 + part;
        }
      }
    }
    double ecoulg = ewald1eng + e2 + e3, evdwg = ev + elrc0;
    spenergy = (ecoulg + evdwg) / sys.engunit;
  } else {
    spenergy = 0.0;
  }
  dlpeng = (ewald1eng + ewald1sum + e2 + ev + elrc0 + e3) / sys.engunit;
  return 0;
}

int Chain::start_server() {
  cudaError_t e = cudaStreamSynchronize(st);  // work on the chain's stream (and its updates) is done
  if (e != cudaSuccess) return sync_error(e);
  st_dirty = false;
  srv_words[0] = srv_words[1] = 0;
  *(volatile int*)&mb->quit = 0;
  h_fl->done = (unsigned long long)pass_seq_done;
  h_fl->go = (unsigned long long)pass_seq_done;
  h_fl->stop = 0;
  h_fl->exit_count = 0;
  e = cudaMemcpyAsync(d_fl, h_fl, sizeof(PassServerFlags), cudaMemcpyHostToDevice, srv_st);
  if (e == cudaSuccess) e = cudaMemsetAsync(W.counter, 0, sizeof(unsigned), srv_st);
  if (e != cudaSuccess) return sync_error(e);
  // 20 ms without a pass end the kernel
  e = launch_pass_server(dsys.view, mb, d_fl, srv_words, W, (long long)pass_seq_done, 20000000LL, srv_st);
  if (e != cudaSuccess) {
    // the blocks cannot all be resident at once (the GPU is busy): passes launch one by one
    cudaGetLastError();
    e = cudaStreamSynchronize(srv_st);
    if (e != cudaSuccess) return sync_error(e);
    use_server = false;
    return 0;
  }
  srv_live = true;
  srv_launches++;
  return 0;
}

int Chain::stop_server() {
  if (!srv_live) return 0;
  *(volatile int*)&mb->quit = 1;
  cudaError_t e = cudaStreamSynchronize(srv_st);  // block 0 sees the flag at its next poll
  srv_live = false;
  *(volatile int*)&mb->quit = 0;
  if (e != cudaSuccess) return sync_error(e);
  return 0;
}

// One pass through the resident kernel: the pass goes into the mailbox, then its number; the
// kernel publishes the energies and then the number, as the one-launch kernel does.  A kernel
// that ended meanwhile (idle limit reached as the pass was posted) is started again and picks
// the posted pass up.
int Chain::pass_resident(const PassArgs& A, double out[3]) {
  if (st_dirty) {
    cudaError_t e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return sync_error(e);
    st_dirty = false;
  }
  if (!srv_live) {
    int rc = start_server();
    if (rc) return rc;
    if (!srv_live) return 1;  // not available: the caller launches the pass
  }
  PassArgsT<kSmallPassSites>& B = mb->A;
  std::memcpy(&B, &A, offsetof(PassArgs, x));
  const int nsite = A.nold + A.nnew;
  for (int i = 0; i < nsite; i++) {
    B.x[i] = A.x[i];
    B.y[i] = A.y[i];
    B.z[i] = A.z[i];
    B.q[i] = A.q[i];
    B.type[i] = A.type[i];
  }
  B.pc = A.pc;
  mb->G = guest_view();
  mb->sk = sk;
  mb->sk_new = sk_new;
  std::atomic_thread_fence(std::memory_order_release);
  *(volatile long long*)&mb->cmd = (long long)A.seq;
  volatile double* flag = W.result + 3;
  for (int restarts = 0;;) {
    long long spins = 0;
    while (*flag != A.seq && !*(volatile int*)&srv_words[0] && ++spins < 400000000LL) {
    }
    std::atomic_thread_fence(std::memory_order_acquire);
    if (*flag == A.seq) break;
    // the kernel ended without the pass, or nothing came back in time: end it, start it again
    *(volatile int*)&mb->quit = 1;
    cudaError_t e = cudaStreamSynchronize(srv_st);
    srv_live = false;
    *(volatile int*)&mb->quit = 0;
    if (e != cudaSuccess) return sync_error(e);
    if (*flag == A.seq) break;
    if (srv_words[1] || ++restarts > 3) return -13;  // a wait inside the kernel ran out
    int rc = start_server();
    if (rc) return rc;
    if (!srv_live) return -13;
  }
  out[0] = W.result[0];
  out[1] = W.result[1];
  out[2] = W.result[2];
  srv_passes++;
  return 0;
}

int Chain::pass(int move, int g, int mol, const double* old_xyz, const double* new_xyz, double out[3]) {
  PassArgs A;
  std::memset(&A, 0, sizeof(A));
  const GuestSpecies& G = sys.deck.guests[g];
  const Species& s = sp[g];
  A.move = move;
  A.nbk = pass_recip_blocks(dsys.view);
  A.do_real = 1;
  A.nold = (move == kInsert) ? 0 : s.nsite;
  A.nnew = (move == kDelete) ? 0 : s.nsite;
  A.ex_lo = A.ex_hi = -1;
  if (mol >= 0) {
    A.ex_lo = s.seg_off + mol * s.nsite;
    A.ex_hi = A.ex_lo + s.nsite;
  }
  A.engsic = sys.engsic[g];
  int w = 0;
  for (int i = 0; i < A.nold; i++, w++) {
    A.x[w] = old_xyz[3 * i];
    A.y[w] = old_xyz[3 * i + 1];
    A.z[w] = old_xyz[3 * i + 2];
    A.q[w] = G.charge[i];
    A.type[w] = (unsigned char)G.type[i];
  }
  for (int i = 0; i < A.nnew; i++, w++) {
    A.x[w] = new_xyz[3 * i];
    A.y[w] = new_xyz[3 * i + 1];
    A.z[w] = new_xyz[3 * i + 2];
    A.q[w] = G.charge[i];
    A.type[w] = (unsigned char)G.type[i];
  }
  if (profile && !ev0) {
    cudaEventCreate(&ev0);
    cudaEventCreate(&ev1);
  }
  if (profile) cudaEventRecord(ev0, st);
  pass_seq += 1.0;
  A.seq = pass_seq;
  take_pending(A);
  if (use_server && !profile && A.nold + A.nnew <= kSmallPassSites) {
    int rc = pass_resident(A, out);
    if (rc <= 0) {
      if (rc == 0) {
        passes++;
        pass_seq_done = pass_seq;
      }
      return rc;
    }
  } else {
    int rc = stop_server();
    if (rc) return rc;
  }
  cudaError_t e = launch_pass(dsys.view, guest_view(), A, sk, sk_new, W, st);
  if (profile) cudaEventRecord(ev1, st);
  if (e == cudaSuccess && !profile) {
    // the kernel writes its energies and then this pass's sequence number into pinned host memory;
    // waiting for the number is quicker than synchronising the stream.  The wait is bounded (well
    // over a second), after which the stream is synchronised, which also reports a failed kernel.
    volatile double* flag = W.result + 3;
    long long spins = 0;
    while (*flag != pass_seq && ++spins < 400000000LL) {
    }
    // the energies were written before the number: read them only after the number (acquire)
    std::atomic_thread_fence(std::memory_order_acquire);
    if (*flag != pass_seq) e = cudaStreamSynchronize(st);
  } else if (e == cudaSuccess) {
    e = cudaStreamSynchronize(st);  // profiled passes: the events need the stream
  }
  if (e != cudaSuccess) return sync_error(e);
  if (profile) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ev0, ev1);
    pass_ms += ms;
    pass_timed++;
  }
  out[0] = W.result[0];
  out[1] = W.result[1];
  out[2] = W.result[2];
  passes++;
  pass_seq_done = pass_seq;
  return 0;
}

void Chain::take_pending(PassArgs& A) {
  if (pend_live) {
    A.pc = pend;
    pend_live = false;
  } else {
    A.pc.op = 0;
    A.pc.seg = -1;
  }
}

int Chain::flush_commit() {
  if (!pend_live) return 0;
  if (int rc0 = stop_server()) return rc0;  // nothing else runs beside the resident kernel
  pend_live = false;
  CommitArgs C;
  std::memset(&C, 0, sizeof(C));
  C.op = pend.op;
  C.lo = pend.lo;
  C.ns = pend.ns;
  C.seg_end = pend.seg_end;
  for (int i = 0; i < pend.ns && pend.op != kDelete; i++) {
    C.x[i] = pend.site[i].x;
    C.y[i] = pend.site[i].y;
    C.z[i] = pend.site[i].z;
    C.q[i] = pend.site[i].w;
    C.type[i] = pend.type[i];
  }
  cudaError_t e = launch_commit(0, sk, sk_new, C, gsite, gtype, st);  // guest sites only
  if (e != cudaSuccess) return sync_error(e);
  commits++;
  return 0;
}

int Chain::commit(int move, int g, int mol, const double* new_xyz) {
  Species& s = sp[g];
  const GuestSpecies& G = sys.deck.guests[g];
  if (move == kInsert && (s.nmol + 1) * s.nsite > s.cap_sites) return -75;
  int rc = flush_commit();  // an update still pending is written first
  if (rc) return rc;
  std::swap(sk, sk_new);  // S_new of the pass becomes S(k); the old buffer takes the next S_new
  PendingCommit& P = pend;
  P.op = move;
  P.seg = g;
  P.ns = s.nsite;
  P.lo = s.seg_off + (move == kInsert ? s.nmol : mol) * s.nsite;
  P.seg_end = s.seg_off + s.nmol * s.nsite;
  if (move != kDelete)
    for (int i = 0; i < s.nsite && i < kMaxPendSites; i++) {
      P.site[i] = make_double4(new_xyz[3 * i], new_xyz[3 * i + 1], new_xyz[3 * i + 2], G.charge[i]);
      P.type[i] = G.type[i];
    }
  pend_live = true;
  if (s.nsite > kMaxPendSites) {
    // too many sites to carry in the next pass's arguments: written now
    CommitArgs C;
    std::memset(&C, 0, sizeof(C));
    C.op = move;
    C.ns = s.nsite;
    C.lo = P.lo;
    C.seg_end = P.seg_end;
    if (move != kDelete)
      for (int i = 0; i < s.nsite; i++) {
        C.x[i] = new_xyz[3 * i];
        C.y[i] = new_xyz[3 * i + 1];
        C.z[i] = new_xyz[3 * i + 2];
        C.q[i] = G.charge[i];
        C.type[i] = G.type[i];
      }
    pend_live = false;
    if (int rc0 = stop_server()) return rc0;
    cudaError_t e = launch_commit(0, sk, sk_new, C, gsite, gtype, st);
    if (e != cudaSuccess) return sync_error(e);
    commits++;
  }
  // host mirror (framwkxxx updates of gcmc.f:966-970, 1134-1138, 1352-1357)
  int n3 = 3 * s.nsite;
  if (move == kInsert) {
    s.xyz.insert(s.xyz.end(), new_xyz, new_xyz + n3);
    s.nmol++;
    totatm += s.nsite;
  } else if (move == kDelete) {
    s.xyz.erase(s.xyz.begin() + (size_t)mol * n3, s.xyz.begin() + (size_t)(mol + 1) * n3);
    s.nmol--;
    totatm -= s.nsite;
  } else {
    std::copy(new_xyz, new_xyz + n3, s.xyz.begin() + (size_t)mol * n3);
  }
  return 0;
}

// One iteration of the move loop (gcmc.f:589-1380 + rolling statistics 1814-1860).
int Chain::step(MoveRecord* rec) {
  const InputDeck& d = sys.deck;
  const int ng = (int)sp.size();
  gcmccount++;
  if (gcmccount % 400 == 0) {
    int totalguests = 0;
    for (auto& s : sp) totalguests += s.nmol;
    if (production) {
      if (d.mcsteps < 0) {
        for (int t = 4; t > 0; t--) tick_tock[t] = tick_tock[t - 1];
        tick_tock[0] = !(prodcount < (long long)(-d.mcsteps) * (totalguests + 1));
        bool all = true;
        for (bool b : tick_tock) all = all && b;
        if (all) lgchk = false;
      } else if (prodcount >= d.mcsteps) {
        lgchk = false;
      }
    } else {
      if (despre > 0) {  // pressure equilibration (gcmc.f:637-696)
        for (int t = 4; t > 0; t--) tick_tock[t] = tick_tock[t - 1];
        tick_tock[0] = !(prodcount < (long long)(-d.eqsteps) * (totalguests + 1) / 4);
        if (tick_tock[0])
          pressure_adjust(ng, gstpress.data(), chainstats.data() + 1, 14, d.adspres.data(), d.adsguen.data(), d.packf,
                          sys.cell.volm, d.temp, presrate, despre, gcmccount, prodcount, d.eqsteps);
      }
      if (d.eqsteps > 0) {
        if (gcmccount >= d.eqsteps && despre == 0) production = true;
      } else if (d.eqsteps < 0) {
        for (int t = 4; t > 0; t--) tick_tock[t] = tick_tock[t - 1];
        tick_tock[0] = !((long long)gcmccount < (long long)(-d.eqsteps) * (totalguests + 1));
        if (despre > 0) tick_tock[0] = false;
        bool all = true;
        for (bool b : tick_tock) all = all && b;
        if (all) {
          production = true;
          for (bool& b : tick_tock) b = false;
        }
      }
    }
  }
  int g = 0;
  if (ng > 1) g = (int)std::floor(duni_next(rng) * ng);
  double randmov = duni_next(rng);
  const std::array<double, 9>& c = sys.mvcum[g];
  int mtype;
  if (randmov < c[0]) mtype = kInsert;
  else if (randmov < c[1]) mtype = kDelete;
  else if (randmov < c[2]) mtype = kDisplace;
  else if (randmov < c[3]) mtype = kJump;
  else if (randmov < c[5]) mtype = kNoop;  // flex, swap (gcmc.f:1789-1795)
  else if (randmov < c[6]) mtype = kTranslate;
  else if (randmov < c[7]) mtype = kRotate;
  else if (randmov < c[8]) mtype = kMultiJump;
  else mtype = kDisplace;
  Species& s = sp[g];
  const GuestSpecies& G = d.guests[g];
  const int natms = s.nsite, nmols = s.nmol;
  // guest geometries before the move (gcmc.f:785-792, hisarchive 2491-2517)
  if (d.nhis != 0 && gcmccount % std::abs(d.nhis) == 0 && !his_f.empty() && (d.nhis < 0 || prodcount > 0))
    for (int k = 0; k < ng; k++) {
      const GuestSpecies& H = d.guests[k];
      std::fprintf(his_f[k], "%6d\nstep %7d\n", sp[k].nmol * sp[k].nsite, gcmccount);
      for (int i = 0, a = 0; i < sp[k].nmol; i++)
        for (int j = 0; j < sp[k].nsite; j++, a++)
          std::fprintf(his_f[k], "  %c%16.6f%16.6f%16.6f\n", H.site_name[j].empty() ? ' ' : H.site_name[j][0],
                       sp[k].xyz[3 * a], sp[k].xyz[3 * a + 1], sp[k].xyz[3 * a + 2]);
    }
  // step-size adaptation (gcmc.f:794-834), applied on every iteration whose counter sits on
  // a multiple of 50/100
  if (nmols >= 1 && disp_count[g] >= 1) {
    if (disp_count[g] % 100 == 0) {
      if ((accept_disp[g] / (double)disp_count[g]) > d.disp_ratio[g]) delrdisp[g] = delrdisp[g] * 1.05;
      else if (delrdisp[g] > kDelrMin) delrdisp[g] = delrdisp[g] * 0.95;
    } else if (disp_count[g] % 50 == 0) {
      if ((accept_disp[g] / (double)disp_count[g]) > d.disp_ratio[g]) rotangle = rotangle * 1.05;
      else if (rotangle > kMinAngle) rotangle = rotangle * 0.95;
    }
  }
  if (nmols >= 1 && tran_count[g] >= 1 && tran_count[g] % 100 == 0) {
    if ((accept_tran[g] / (double)tran_count[g]) > d.tran_ratio[g]) tran_delr[g] = tran_delr[g] * 1.05;
    else if (tran_delr[g] > kDelrMin) tran_delr[g] = tran_delr[g] * 0.95;
  }
  if (nmols >= 1 && rota_count >= 1 && rota_count % 100 == 0) {
    if ((accept_rota / (double)rota_count) > d.rota_ratio) rota_rotangle = rota_rotangle * 1.05;
    else if (rota_rotangle > kMinAngle) rota_rotangle = rota_rotangle * 0.95;
  }
  if (nmols == 0 || (nmols == 1 && mtype == kMultiJump)) mtype = kInsert;  // gcmc.f:837-847
  MoveRecord R;
  std::memset(&R, 0, sizeof(R));
  R.step = gcmccount;
  R.iguest = g;
  R.mtype = mtype;
  bool accepted = false;
  double e[3] = {0, 0, 0}, ewld3 = 0, delrc = 0, estep = 0, rande = -1;
  double oldx[3 * kMaxGuestSites], newx[3 * kMaxGuestSites];
  delE[g] = 0.0;
  last_guest = g;
  int rc = 0;
  if (mtype == kInsert) {
    ins_count++;
    if ((totatm - framatm) + natms >= d.maxguest) return -75;
    double r[7];
    for (int i = 0; i < 7; i++) r[i] = duni_next(rng);
    double x[kMaxGuestSites], y[kMaxGuestSites], z[kMaxGuestSites];
    trial_insert(sys.cell, G.tx.data(), G.ty.data(), G.tz.data(), natms, r, x, y, z);
    for (int i = 0; i < natms; i++) {
      newx[3 * i] = x[i];
      newx[3 * i + 1] = y[i];
      newx[3 * i + 2] = z[i];
    }
    if ((rc = pass(kInsert, g, -1, nullptr, newx, e))) return rc;
    for (int i = 0; i < natms; i++) numtyp[G.type[i]]++;
    delrc = lrc_energy(sys, numtyp, numfrz) - elrc;
    ewld3 = sys.ewald3en[g];
    estep = (e[0] + e[1] + ewld3 + e[2] + delrc) / sys.engunit;
    rande = duni_next(rng);
    accepted = accept_move(estep, rande, sys.statvolm, gstpress[g], nmols, d.temp, sys.beta, kInsert);
    if (accepted) {
      delE[g] = estep;
      accept_ins++;
      if ((rc = commit(kInsert, g, -1, newx))) return rc;
      elrc = elrc + delrc;
      energy[g] += delE[g];
    } else {
      for (int i = 0; i < natms; i++) numtyp[G.type[i]]--;
    }
  } else if (mtype == kDelete) {
    del_count++;
    int randchoice = (int)std::floor(duni_next(rng) * nmols) + 1;
    R.randchoice = randchoice;
    int mol = randchoice - 1;
    std::copy(s.xyz.begin() + (size_t)mol * 3 * natms, s.xyz.begin() + (size_t)(mol + 1) * 3 * natms, oldx);
    for (int i = 0; i < natms; i++) numtyp[G.type[i]]--;
    delrc = lrc_energy(sys, numtyp, numfrz) - elrc;
    if ((rc = pass(kDelete, g, mol, oldx, nullptr, e))) return rc;
    ewld3 = sys.ewald3en[g];
    estep = (e[0] - e[1] - ewld3 - e[2] + delrc) / sys.engunit;
    rande = duni_next(rng);
    accepted = accept_move(estep, rande, sys.statvolm, gstpress[g], nmols, d.temp, sys.beta, kDelete);
    if (accepted) {
      delE[g] = estep;
      accept_del++;
      if ((rc = commit(kDelete, g, mol, nullptr))) return rc;
      elrc = elrc + delrc;
      energy[g] += delE[g];
    } else {
      for (int i = 0; i < natms; i++) numtyp[G.type[i]]++;
    }
  } else if (mtype == kJump) {
    // long jump (gcmc.f:1389-1547): choice first, then the seven draws of random_jump
    jump_count++;
    int randchoice = (int)std::floor(duni_next(rng) * nmols) + 1;
    R.randchoice = randchoice;
    int mol = randchoice - 1;
    std::copy(s.xyz.begin() + (size_t)mol * 3 * natms, s.xyz.begin() + (size_t)(mol + 1) * 3 * natms, oldx);
    double r[7];
    for (int i = 0; i < 7; i++) r[i] = duni_next(rng);
    double x[kMaxGuestSites], y[kMaxGuestSites], z[kMaxGuestSites];
    for (int i = 0; i < natms; i++) {
      x[i] = oldx[3 * i];
      y[i] = oldx[3 * i + 1];
      z[i] = oldx[3 * i + 2];
    }
    trial_jump(sys.cell, G.mass.data(), natms, r, x, y, z);
    for (int i = 0; i < natms; i++) {
      newx[3 * i] = x[i];
      newx[3 * i + 1] = y[i];
      newx[3 * i + 2] = z[i];
    }
    if ((rc = pass(kDisplace, g, mol, oldx, newx, e))) return rc;
    estep = (e[0] + e[1] + e[2]) / sys.engunit;
    if (estep < 0.0) {
      accepted = true;
    } else {
      rande = duni_next(rng);
      accepted = accept_move(estep, rande, sys.statvolm, gstpress[g], nmols, d.temp, sys.beta, kDisplace);
    }
    if (accepted) {
      delE[g] = estep;
      accept_jump++;
      if ((rc = commit(kDisplace, g, mol, newx))) return rc;
      energy[g] += delE[g];
    }
  } else if (mtype == kMultiJump) {
    // two distinct molecules jump one after the other (gcmc.f:1557-1785); the first jump is
    // committed before the second is evaluated, one test decides on the summed change and a
    // rejection puts the first molecule and S(k) back
    jump_count++;
    const double origenergy = energy[g];
    cudaError_t ce = cudaMemcpyAsync(sk_save, sk, sizeof(double2) * std::max(sys.K, 1), cudaMemcpyDeviceToDevice, st);
    if (ce != cudaSuccess) return sync_error(ce);
    st_dirty = true;
    int first = 0, mol = -1;
    double first_old[3 * kMaxGuestSites];
    for (int mv = 1; mv <= 2; mv++) {
      int randchoice;
      do {  // a molecule that has not jumped in this move
        randchoice = (int)std::floor(duni_next(rng) * nmols) + 1;
      } while (randchoice == first);
      if (mv == 1) first = randchoice;
      R.randchoice = randchoice;
      mol = randchoice - 1;
      std::copy(s.xyz.begin() + (size_t)mol * 3 * natms, s.xyz.begin() + (size_t)(mol + 1) * 3 * natms, oldx);
      double r[7];
      for (int i = 0; i < 7; i++) r[i] = duni_next(rng);
      double x[kMaxGuestSites], y[kMaxGuestSites], z[kMaxGuestSites];
      for (int i = 0; i < natms; i++) {
        x[i] = oldx[3 * i];
        y[i] = oldx[3 * i + 1];
        z[i] = oldx[3 * i + 2];
      }
      trial_jump(sys.cell, G.mass.data(), natms, r, x, y, z);
      for (int i = 0; i < natms; i++) {
        newx[3 * i] = x[i];
        newx[3 * i + 1] = y[i];
        newx[3 * i + 2] = z[i];
      }
      if ((rc = pass(kDisplace, g, mol, oldx, newx, e))) return rc;
      estep = estep + (e[0] + e[1] + e[2]) / sys.engunit;
      if (mv == 1) {
        std::copy(oldx, oldx + 3 * natms, first_old);
        if ((rc = commit(kDisplace, g, mol, newx))) return rc;
        delE[g] = estep;
        energy[g] = origenergy + delE[g];
      }
    }
    if (estep < 0.0) {
      accepted = true;
    } else {
      rande = duni_next(rng);
      accepted = accept_move(estep, rande, sys.statvolm, gstpress[g], nmols, d.temp, sys.beta, kDisplace);
    }
    if (accepted) {
      delE[g] = estep;
      accept_jump++;
      if ((rc = commit(kDisplace, g, mol, newx))) return rc;
      energy[g] = origenergy + delE[g];
    } else {
      delE[g] = 0.0;
      // S(k) back to its state before the move; the first molecule back to its old sites
      ce = cudaMemcpyAsync(sk_new, sk_save, sizeof(double2) * std::max(sys.K, 1), cudaMemcpyDeviceToDevice, st);
      if (ce != cudaSuccess) return sync_error(ce);
      st_dirty = true;
      if ((rc = commit(kDisplace, g, first - 1, first_old))) return rc;
      energy[g] = origenergy;
    }
  } else if (mtype == kNoop) {
    accepted = last_accepted;  // the reference leaves `accepted` as the last move set it
  } else {
    double r[7], dis_delr, dis_rot;
    if (mtype == kTranslate) {
      tran_count[g]++;
      r[0] = duni_next(rng);
      r[1] = duni_next(rng);
      r[2] = duni_next(rng);
      r[3] = r[4] = r[5] = r[6] = 0.0;
      dis_delr = tran_delr[g];
      dis_rot = 0.0;
    } else if (mtype == kRotate) {
      rota_count++;
      r[0] = r[1] = r[2] = 0.5;
      for (int i = 3; i < 7; i++) r[i] = duni_next(rng);
      dis_delr = 0.0;
      dis_rot = rota_rotangle;
    } else {
      disp_count[g]++;
      for (int i = 0; i < 7; i++) r[i] = duni_next(rng);
      dis_delr = delrdisp[g];
      dis_rot = rotangle;
    }
    int randchoice = (int)std::floor(duni_next(rng) * nmols) + 1;
    R.randchoice = randchoice;
    int mol = randchoice - 1;
    std::copy(s.xyz.begin() + (size_t)mol * 3 * natms, s.xyz.begin() + (size_t)(mol + 1) * 3 * natms, oldx);
    double x[kMaxGuestSites], y[kMaxGuestSites], z[kMaxGuestSites];
    for (int i = 0; i < natms; i++) {
      x[i] = oldx[3 * i];
      y[i] = oldx[3 * i + 1];
      z[i] = oldx[3 * i + 2];
    }
    trial_displace(sys.cell, G.mass.data(), natms, dis_delr, dis_rot, r, x, y, z);
    for (int i = 0; i < natms; i++) {
      newx[3 * i] = x[i];
      newx[3 * i + 1] = y[i];
      newx[3 * i + 2] = z[i];
    }
    if ((rc = pass(kDisplace, g, mol, oldx, newx, e))) return rc;
    estep = (e[0] + e[1] + e[2]) / sys.engunit;
    if (estep < 0.0) {
      accepted = true;
    } else {
      rande = duni_next(rng);
      accepted = accept_move(estep, rande, sys.statvolm, gstpress[g], nmols, d.temp, sys.beta, kDisplace);
    }
    if (accepted) {
      delE[g] = estep;
      if (mtype == kTranslate) accept_tran[g]++;
      else if (mtype == kRotate) accept_rota++;
      else accept_disp[g]++;
      if ((rc = commit(kDisplace, g, mol, newx))) return rc;
      energy[g] += delE[g];
    }
  }
  last_accepted = accepted;
  // running loading while the pressures equilibrate (gcmc.f:1796-1808)
  if (!production && despre > 0 && ((d.laccsample && accepted) || !d.laccsample)) {
    prodcount++;
    for (int i = 0; i < ng; i++) {
      double* a = chainstats.data() + 14 * i + 1;
      *a = *a + ((double)(float)sp[i].nmol - *a) / (double)prodcount;
    }
  }
  if (production && ((d.laccsample && accepted) || !d.laccsample)) {
    prodcount++;
    win.rollcount++;
    chainstats[0] = (double)prodcount;
    double pc = (double)prodcount;
    for (int i = 0; i < ng; i++) {
      double dm = (double)(float)sp[i].nmol, m2 = dm * dm, en = energy[i], e2 = en * en;
      if (prodcount <= kSampleCap + 1) {  // gasmol / gaseng (gcmc.f:1824-1827)
        gasmol[(size_t)i * kSampleCap + prodcount - 1] = dm;
        gaseng[(size_t)i * kSampleCap + prodcount - 1] = en;
      }
      double* cs = chainstats.data() + 14 * i;
      cs[1] = cs[1] + (dm - cs[1]) / pc;
      cs[2] = cs[2] + (en - cs[2]) / pc;
      cs[3] = cs[3] + (en * dm - cs[3]) / pc;
      cs[4] = cs[4] + (m2 - cs[4]) / pc;
      cs[5] = cs[5] + (e2 - cs[5]) / pc;
      window_sample(win, i, dm, en, mtype == kInsert && g == i && accepted, delE[i], d.temp, accept_ins, cs + 1);
    }
  }
  if (production && (prodcount % d.nwind == 0 || !lgchk))
    window_close(win, ng, d.nwind, d.temp, [this](int i) { return (const double*)chainstats.data() + 14 * i + 1; });
  if (production && !prob.empty()) store_prob();  // gcmc.f:1929-1931, every production move
  // numguests.out (gcmc.f:1937-1951): only the moved species carries its dE and move flags
  if (!numg_f.empty() && gcmccount % d.nnumg == 0) {
    int fl[6] = {0, 0, 0, 0, 0, 0};
    if (mtype == kInsert) fl[0] = 1;
    else if (mtype == kDelete) fl[1] = 1;
    else if (mtype == kDisplace) fl[2] = 1;
    else if (mtype == kTranslate) fl[2] = 2;
    else if (mtype == kRotate) fl[2] = 3;
    else if (mtype == kJump) fl[3] = 1;
    else if (mtype == kMultiJump) fl[3] = 2;
    for (int i = 0; i < ng; i++) {
      const bool me = i == g;
      std::fprintf(numg_f[i], "%9d%7d%20.6f%20.6f%4d%4d%4d%4d%4d%4d\n", gcmccount, sp[i].nmol, energy[i],
                   me ? delE[i] : 0.0, me ? fl[0] : 0, me ? fl[1] : 0, me ? fl[2] : 0, me ? fl[3] : 0,
                   me ? fl[4] : 0, me ? fl[5] : 0);
    }
  }
  R.accepted = accepted;
  R.nmols_after = s.nmol;
  R.ewld1 = e[0];
  R.ewld2 = (mtype == kInsert || mtype == kDelete) ? e[1] : e[1];
  R.ewld3 = ewld3;
  R.vdw = e[2];
  R.delrc = delrc;
  R.estep = estep;
  R.rande = rande;
  R.energy_after = energy[g];
  if (rec) *rec = R;
  return 0;
}

}  // namespace fmc
