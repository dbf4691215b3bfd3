// extern "C" boundary (include/fastmc_b200.h) over fmc::Chain.
#include <cstdio>
#include <cstring>
#include <string>

#include "../../include/fastmc_b200.h"
#include "fmc_chain.h"
#include "fmc_desc.h"
#include "fmc_restart.h"

struct fmc_chain {
  fmc::Chain impl;
  // displace pass 1 of the drop-in ewald1_guest call stores the molecule's old sites here
  int pending_g = -1, pending_n = 0;
  double pending_old[3 * fmc::kMaxGuestSites];
};

namespace {
thread_local std::string g_err;
int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}
#define CHECK_CHAIN(c) \
  if (!(c)) return fail(-1, "null chain handle")
}  // namespace

namespace fmc {
void set_last_error(const std::string& msg) { g_err = msg; }
}  // namespace fmc

extern "C" {

int fmc_version(void) { return 10400; }

const char* fmc_last_error(void) { return g_err.c_str(); }

int fmc_chain_open_node(const char* dir, const int* seed, int device, int idnode, fmc_chain** out) {
  if (!dir || !seed || !out) return fail(-1, "null argument");
  *out = nullptr;
  fmc_chain* c = new fmc_chain();
  std::string err;
  int rc = c->impl.open(dir, seed, device, err);
  // CONTROL `restart`: this node's branch REVIVE, read after duni is seeded as gcmc.f:334-394
  // does (a single point never continues a run)
  const fmc::InputDeck& d = c->impl.sys.deck;
  if (!rc && d.lrestart && !d.lspe) {
    fmc::BranchChoice b;
    rc = fmc::choose_branch(dir, idnode, b, err);
    fmc::Revive r;
    if (!rc && !b.revive.empty()) rc = fmc::read_revive(b.revive, d, r, err);
    if (!rc && !b.revive.empty()) rc = c->impl.restart(r, err);
  }
  if (rc) {
    delete c;
    return fail(rc, err);
  }
  *out = c;
  return 0;
}

int fmc_chain_open(const char* dir, const int* seed, int device, fmc_chain** out) {
  return fmc_chain_open_node(dir, seed, device, 0, out);
}

int fmc_restart_branch(const char* workdir, int idnode, char* revive_path, int revive_cap, char* outdir,
                       int outdir_cap, int* prevnodes) {
  if (!workdir || (!revive_path && revive_cap) || (!outdir && outdir_cap)) return fail(-1, "bad arguments");
  fmc::BranchChoice b;
  std::string err;
  if (int rc = fmc::choose_branch(workdir, idnode, b, err)) return fail(rc, err);
  if ((revive_path && (int)b.revive.size() >= revive_cap) || (outdir && (int)b.outdir.size() >= outdir_cap))
    return fail(-1, "path buffer too small");
  if (revive_path) std::memcpy(revive_path, b.revive.c_str(), b.revive.size() + 1);
  if (outdir) std::memcpy(outdir, b.outdir.c_str(), b.outdir.size() + 1);
  if (prevnodes) *prevnodes = b.prevnodes;
  return b.revive.empty() ? 0 : 1;
}

void fmc_chain_close(fmc_chain* c) { delete c; }

int fmc_chain_create(const fmc_system_desc* desc, const int* seed, int device, fmc_chain** out) {
  if (!desc || !seed || !out) return fail(-1, "null argument");
  *out = nullptr;
  fmc::InputDeck deck;
  std::string err;
  int rc = fmc::deck_from_desc(*desc, deck, err);
  if (rc) return fail(rc, err);
  fmc::HostSystem h;
  rc = fmc::build_host_system(deck, h, err);
  if (rc) return fail(rc, err);
  fmc_chain* c = new fmc_chain();
  rc = c->impl.open_prepared(std::move(h), seed, device, err);
  if (rc) {
    delete c;
    return fail(rc, err);
  }
  *out = c;
  return 0;
}

int fmc_deck_describe(const char* dir, fmc_system_desc* out) {
  if (!dir || !out) return fail(-1, "null argument");
  std::string err;
  int rc = fmc::describe_deck(dir, *out, err);
  if (rc) return fail(rc, err);
  return 0;
}

void fmc_desc_free(fmc_system_desc* desc) {
  if (desc && desc->owner) fmc::free_desc(*desc);
}

int fmc_desc_sizes(int* out) {
  if (!out) return fail(-1, "null argument");
  out[0] = (int)sizeof(fmc_system_desc);
  out[1] = (int)sizeof(fmc_guest_desc);
  out[2] = (int)sizeof(fmc_vdw_desc);
  return 0;
}

int fmc_chain_info(fmc_chain* c, int* ints, double* dbls) {
  CHECK_CHAIN(c);
  const fmc::Chain& C = c->impl;
  const fmc::HostSystem& S = C.sys;
  int nv = S.nvox[0] * S.nvox[1] * S.nvox[2];
  int iv[16] = {S.cell.imcon, S.deck.kmax[0], S.deck.kmax[1], S.deck.kmax[2], S.K, C.totatm, (int)C.sp.size(),
                S.ntypes, S.mxgrid, S.nf, C.gcmccount, nv, C.gcap, 0, 0, 0};
  double dv[16] = {S.alpha, S.rcut, S.deck.delr, S.cell.volm, S.engunit, S.deck.temp, S.beta, S.drewd, S.dlrpot,
                   C.spenergy, C.dlpeng, C.ewald1sum, C.elrc, C.energy.empty() ? 0.0 : C.energy[0], S.statvolm, 0.0};
  if (ints) std::memcpy(ints, iv, sizeof(iv));
  if (dbls) std::memcpy(dbls, dv, sizeof(dv));
  return 0;
}

int fmc_ewald1(fmc_chain* c, double* engcpe, int* newld) {
  CHECK_CHAIN(c);
  double e = 0.0;
  int rc = c->impl.full_recip(&e);
  if (rc) return fail(rc, "ewald1 failed on the device");
  if (engcpe) *engcpe = e;
  if (newld) *newld = c->impl.sys.K;
  return 0;
}

int fmc_ewald1_guest(fmc_chain* c, int iguest, int natms, const double* xyz, int move, int pass, double* engcpe) {
  CHECK_CHAIN(c);
  fmc::Chain& C = c->impl;
  if (iguest < 0 || iguest >= (int)C.sp.size()) return fail(-1, "species index out of range");
  if (natms != C.sp[iguest].nsite) return fail(-1, "natms differs from the species' site count");
  double out[3];
  if (move == FMC_DISPLACE && pass == 1) {
    c->pending_g = iguest;
    c->pending_n = natms;
    std::memcpy(c->pending_old, xyz, sizeof(double) * 3 * natms);
    if (engcpe) *engcpe = 0.0;
    return 0;
  }
  fmc::PassArgs A;
  std::memset(&A, 0, sizeof(A));
  const fmc::GuestSpecies& G = C.sys.deck.guests[iguest];
  A.move = move == FMC_DISPLACE ? fmc::kDisplace : (move == FMC_DELETE ? fmc::kDelete : fmc::kInsert);
  if (A.move == fmc::kDisplace && c->pending_g != iguest) return fail(-1, "displace pass 2 without pass 1");
  A.nbk = fmc::pass_recip_blocks(C.dsys.view);
  A.do_real = 0;
  A.nold = A.move == fmc::kInsert ? 0 : natms;
  A.nnew = A.move == fmc::kDelete ? 0 : natms;
  A.ex_lo = A.ex_hi = -1;
  A.engsic = C.sys.engsic[iguest];
  const double* olds = A.move == fmc::kDisplace ? c->pending_old : xyz;
  int w = 0;
  for (int i = 0; i < A.nold; i++, w++) {
    A.x[w] = olds[3 * i];
    A.y[w] = olds[3 * i + 1];
    A.z[w] = olds[3 * i + 2];
    A.q[w] = G.charge[i];
    A.type[w] = (unsigned char)G.type[i];
  }
  for (int i = 0; i < A.nnew; i++, w++) {
    A.x[w] = xyz[3 * i];
    A.y[w] = xyz[3 * i + 1];
    A.z[w] = xyz[3 * i + 2];
    A.q[w] = G.charge[i];
    A.type[w] = (unsigned char)G.type[i];
  }
  if (int rc0 = C.stop_server()) return fail(rc0, "the resident pass kernel did not end");
  C.take_pending(A);  // an update left by fmc_commit is read through and written by this pass
  cudaError_t e = fmc::launch_pass(C.dsys.view, C.guest_view(), A, C.sk, C.sk_new, C.W, C.st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(C.st);  // the kernel wrote the result to pinned memory
  if (e != cudaSuccess) return fail(-100 - (int)e, cudaGetErrorString(e));
  out[0] = C.W.result[0];
  if (A.move == fmc::kDisplace) c->pending_g = -1;
  if (engcpe) *engcpe = out[0];
  return 0;
}

int fmc_guest_realspace(fmc_chain* c, int iguest, int natms, const double* xyz, int mol, double* ewld2, double* vdw) {
  CHECK_CHAIN(c);
  fmc::Chain& C = c->impl;
  if (iguest < 0 || iguest >= (int)C.sp.size()) return fail(-1, "species index out of range");
  if (natms != C.sp[iguest].nsite) return fail(-1, "natms differs from the species' site count");
  if (mol >= C.sp[iguest].nmol) return fail(-1, "molecule index out of range");
  fmc::PassArgs A;
  std::memset(&A, 0, sizeof(A));
  const fmc::GuestSpecies& G = C.sys.deck.guests[iguest];
  A.move = fmc::kInsert;
  A.nbk = 0;
  A.do_real = 1;
  A.nold = 0;
  A.nnew = natms;
  A.ex_lo = A.ex_hi = -1;
  if (mol >= 0) {
    A.ex_lo = C.sp[iguest].seg_off + mol * natms;
    A.ex_hi = A.ex_lo + natms;
  }
  for (int i = 0; i < natms; i++) {
    A.x[i] = xyz[3 * i];
    A.y[i] = xyz[3 * i + 1];
    A.z[i] = xyz[3 * i + 2];
    A.q[i] = G.charge[i];
    A.type[i] = (unsigned char)G.type[i];
  }
  if (int rc0 = C.stop_server()) return fail(rc0, "the resident pass kernel did not end");
  C.take_pending(A);  // an update left by fmc_commit is read through and written by this pass
  cudaError_t e = fmc::launch_pass(C.dsys.view, C.guest_view(), A, C.sk, C.sk_new, C.W, C.st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(C.st);  // the kernel wrote the result to pinned memory
  if (e != cudaSuccess) return fail(-100 - (int)e, cudaGetErrorString(e));
  if (ewld2) *ewld2 = C.W.result[1];
  if (vdw) *vdw = C.W.result[2];
  return 0;
}

int fmc_commit(fmc_chain* c, int move, int iguest, int mol, const double* xyz) {
  CHECK_CHAIN(c);
  fmc::Chain& C = c->impl;
  if (iguest < 0 || iguest >= (int)C.sp.size()) return fail(-1, "species index out of range");
  int m = move == FMC_DELETE ? fmc::kDelete : (move == FMC_INSERT ? fmc::kInsert : fmc::kDisplace);
  if (m != fmc::kInsert && (mol < 0 || mol >= C.sp[iguest].nmol)) return fail(-1, "molecule index out of range");
  int rc = C.commit(m, iguest, mol, xyz);
  if (rc == -75) return fail(75, "too many atoms in specified system");
  if (rc) return fail(rc, "commit failed on the device");
  cudaError_t e = cudaStreamSynchronize(C.st);
  if (e != cudaSuccess) return fail(-100 - (int)e, cudaGetErrorString(e));
  return 0;
}

int fmc_reject(fmc_chain* c) {
  CHECK_CHAIN(c);
  return 0;
}

namespace {
// x[n], y[n], z[n] -> interleaved x,y,z (the layout of the calls above)
bool interleave(int n, const double* x, const double* y, const double* z, double* out) {
  if (n < 0 || n > fmc::kMaxGuestSites || !x || !y || !z) return false;
  for (int i = 0; i < n; i++) {
    out[3 * i] = x[i];
    out[3 * i + 1] = y[i];
    out[3 * i + 2] = z[i];
  }
  return true;
}
}  // namespace

int fmc_ewald1_guest_xyz(fmc_chain* c, int iguest, int natms, const double* x, const double* y, const double* z,
                         int move, int pass, double* engcpe) {
  double xyz[3 * fmc::kMaxGuestSites];
  if (!interleave(natms, x, y, z, xyz)) return fail(-1, "null coordinate array or site count out of range");
  return fmc_ewald1_guest(c, iguest, natms, xyz, move, pass, engcpe);
}

int fmc_guest_realspace_xyz(fmc_chain* c, int iguest, int natms, const double* x, const double* y, const double* z,
                            int mol, double* ewld2, double* vdw) {
  double xyz[3 * fmc::kMaxGuestSites];
  if (!interleave(natms, x, y, z, xyz)) return fail(-1, "null coordinate array or site count out of range");
  return fmc_guest_realspace(c, iguest, natms, xyz, mol, ewld2, vdw);
}

int fmc_commit_xyz(fmc_chain* c, int move, int iguest, int mol, const double* x, const double* y, const double* z) {
  CHECK_CHAIN(c);
  if (move == FMC_DELETE) return fmc_commit(c, move, iguest, mol, nullptr);
  if (iguest < 0 || iguest >= (int)c->impl.sp.size()) return fail(-1, "species index out of range");
  double xyz[3 * fmc::kMaxGuestSites];
  if (!interleave(c->impl.sp[iguest].nsite, x, y, z, xyz))
    return fail(-1, "null coordinate array or site count out of range");
  return fmc_commit(c, move, iguest, mol, xyz);
}

int fmc_set_guests(fmc_chain* c, int iguest, int nmol, const double* xyz) {
  CHECK_CHAIN(c);
  fmc::Chain& C = c->impl;
  if (iguest < 0 || iguest >= (int)C.sp.size()) return fail(-1, "species index out of range");
  int rc = C.set_guests(iguest, nmol, xyz);
  if (rc == -75) return fail(75, "too many atoms in specified system");
  if (rc) return fail(rc, "guest upload failed");
  rc = C.full_recip(nullptr);
  if (rc) return fail(rc, "ewald1 failed on the device");
  return 0;
}

int fmc_single_point(fmc_chain* c, double* spenergy, double* dlpeng) {
  CHECK_CHAIN(c);
  int rc = c->impl.single_point();
  if (rc) return fail(rc, "single point failed on the device");
  if (spenergy) *spenergy = c->impl.spenergy;
  if (dlpeng) *dlpeng = c->impl.dlpeng;
  return 0;
}

int fmc_chain_resident(fmc_chain* c, int enable, long long* launches, long long* passes) {
  CHECK_CHAIN(c);
  fmc::Chain& C = c->impl;
  if (enable >= 0) {
    if (int rc = C.stop_server()) return fail(rc, "the resident pass kernel did not end");
    C.use_server = enable != 0;
  }
  if (launches) *launches = C.srv_launches;
  if (passes) *passes = C.srv_passes;
  return C.use_server ? 1 : 0;
}

int fmc_get_sk(fmc_chain* c, int pending, double* re, double* im) {
  CHECK_CHAIN(c);
  fmc::Chain& C = c->impl;
  if (int rc0 = C.stop_server()) return fail(rc0, "the resident pass kernel did not end");
  std::vector<double2> h(C.sys.K);
  cudaError_t e = cudaMemcpyAsync(h.data(), pending ? C.sk_new : C.sk, sizeof(double2) * C.sys.K,
                                  cudaMemcpyDeviceToHost, C.st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(C.st);
  if (e != cudaSuccess) return fail(-100 - (int)e, cudaGetErrorString(e));
  for (int k = 0; k < C.sys.K; k++) {
    if (re) re[k] = h[k].x;
    if (im) im[k] = h[k].y;
  }
  return 0;
}

int fmc_kvectors(fmc_chain* c, int* lmn, double* akk) {
  CHECK_CHAIN(c);
  const fmc::HostSystem& S = c->impl.sys;
  for (int k = 0; k < S.K; k++) {
    if (lmn) {
      lmn[3 * k] = S.kl[k];
      lmn[3 * k + 1] = S.km[k];
      lmn[3 * k + 2] = S.kn[k];
    }
    if (akk) akk[k] = S.akk[k];
  }
  return 0;
}

int fmc_run(fmc_chain* c, int nmoves, fmc_move_record* trace) {
  CHECK_CHAIN(c);
  static_assert(sizeof(fmc_move_record) == sizeof(fmc::MoveRecord), "record layout");
  for (int i = 0; i < nmoves; i++) {
    int rc = c->impl.step(trace ? reinterpret_cast<fmc::MoveRecord*>(trace + i) : nullptr);
    if (rc == -75) return fail(75, "too many atoms in specified system");
    if (rc) return fail(rc, "move loop failed");
  }
  return 0;
}

int fmc_guest_coords(fmc_chain* c, int iguest, double* xyz, int* nmol, int* nsite) {
  CHECK_CHAIN(c);
  fmc::Chain& C = c->impl;
  if (iguest < 0 || iguest >= (int)C.sp.size()) return fail(-1, "species index out of range");
  if (nmol) *nmol = C.sp[iguest].nmol;
  if (nsite) *nsite = C.sp[iguest].nsite;
  if (xyz) std::memcpy(xyz, C.sp[iguest].xyz.data(), sizeof(double) * C.sp[iguest].xyz.size());
  return 0;
}

int fmc_revive_write_state(const char* deck_dir, const char* outdir, int production, const int* nmol,
                           const double* guest_xyz, const double* chainstats, const double* energy, double eng) {
  if (!deck_dir || !outdir || !nmol) return fail(-1, "bad arguments");
  fmc::InputDeck d;
  std::string err;
  int rc = fmc::read_input_deck(deck_dir, d, err);
  if (rc) return fail(rc, err);
  const int ng = (int)d.guests.size();
  std::vector<std::vector<double>> xyz(ng);
  size_t off = 0;
  for (int g = 0; g < ng; g++) {
    const size_t n = 3 * (size_t)nmol[g] * d.guests[g].nsite;
    if (n && !guest_xyz) return fail(-1, "guest coordinates missing");
    xyz[g].assign(guest_xyz + off, guest_xyz + off + n);
    off += n;
  }
  std::vector<double> cs(1 + 14 * ng, 0.0), en(ng, 0.0);
  if (chainstats) cs.assign(chainstats, chainstats + cs.size());
  if (energy) en.assign(energy, energy + ng);
  fmc::Revive r = fmc::revive_state(d, production != 0, xyz, cs, en);
  rc = fmc::write_revive(std::string(outdir) + "/REVIVE", r, err);
  if (!rc) rc = fmc::write_revcon(std::string(outdir) + "/REVCON", d, r, eng, err);
  return rc ? fail(rc, err) : 0;
}

int fmc_revive_read(const char* path, const char* deck_dir, int* production, int* nmol, double* guest_xyz,
                    double* chainstats, double* energy, int* natms) {
  if (!path || !deck_dir) return fail(-1, "bad arguments");
  fmc::InputDeck d;
  std::string err;
  int rc = fmc::read_input_deck(deck_dir, d, err);
  if (rc) return fail(rc, err);
  fmc::Revive r;
  rc = fmc::read_revive(path, d, r, err);
  if (rc) return fail(rc, err);
  const auto xyz = fmc::revive_guest_xyz(d, r);
  const int ng = (int)d.guests.size();
  if (production) *production = r.production ? 1 : 0;
  if (natms) *natms = r.natms;
  size_t off = 0;
  for (int g = 0; g < ng; g++) {
    if (nmol) nmol[g] = (int)(xyz[g].size() / (3 * d.guests[g].nsite));
    if (guest_xyz) std::memcpy(guest_xyz + off, xyz[g].data(), sizeof(double) * xyz[g].size());
    off += xyz[g].size();
  }
  if (chainstats) std::memcpy(chainstats, r.chainstats.data(), sizeof(double) * r.chainstats.size());
  if (energy) std::memcpy(energy, r.energy.data(), sizeof(double) * r.energy.size());
  return 0;
}

int fmc_chain_write_revive(fmc_chain* c, const char* outdir) {
  CHECK_CHAIN(c);
  if (!outdir) return fail(-1, "bad arguments");
  fmc::Chain& C = c->impl;
  std::vector<std::vector<double>> xyz;
  for (auto& s : C.sp) xyz.push_back(std::vector<double>(s.xyz.begin(), s.xyz.begin() + 3 * s.nmol * s.nsite));
  fmc::Revive r = fmc::revive_state(C.sys.deck, C.production, xyz, C.chainstats, C.energy);
  std::string err;
  int rc = fmc::write_revive(std::string(outdir) + "/REVIVE", r, err);
  const double eng = C.delE.empty() ? 0.0 : C.delE[C.last_guest];
  if (!rc) rc = fmc::write_revcon(std::string(outdir) + "/REVCON", C.sys.deck, r, eng, err);
  return rc ? fail(rc, err) : 0;
}

int fmc_chain_restart(fmc_chain* c, const char* revive_path) {
  CHECK_CHAIN(c);
  if (!revive_path) return fail(-1, "bad arguments");
  fmc::Revive r;
  std::string err;
  int rc = fmc::read_revive(revive_path, c->impl.sys.deck, r, err);
  if (!rc) rc = c->impl.restart(r, err);
  return rc ? fail(rc, err) : 0;
}

int fmc_atomic_number(double mass) { return fmc::atomic_number(mass); }

int fmc_write_prob_cube(const char* deck_dir, const char* path, const double* grid, long long steps) {
  if (!deck_dir || !path || !grid || steps < 1) return fail(-1, "bad arguments");
  fmc::InputDeck d;
  std::string err;
  int rc = fmc::read_input_deck(deck_dir, d, err);
  if (!rc && d.plots.empty()) {
    rc = -1;
    err = "the deck requests no probability plots";
  }
  if (!rc) rc = fmc::write_prob_cube(path, d, grid, steps, err);
  return rc ? fail(rc, err) : 0;
}

int fmc_write_report(const char* deck_dir, const double* final_stats, const double* seltot, const char* path) {
  if (!deck_dir || !final_stats || !path) return fail(-1, "bad arguments");
  fmc::InputDeck d;
  std::string err;
  int rc = fmc::read_input_deck(deck_dir, d, err);
  if (rc) return fail(rc, err);
  const int ng = (int)d.guests.size();
  if (ng > 4) return fail(-1, "more than 4 guest species");
  fmc::WindowStats W{};
  if (seltot)
    for (int i = 0; i < ng; i++)
      for (int j = 0; j < ng; j++) W.seltot[i][j] = seltot[i * ng + j];
  rc = fmc::write_report(path, d, final_stats, W, d.temp, err);
  return rc ? fail(rc, err) : 0;
}

int fmc_chain_prob(fmc_chain* c, int plot, int* dims, double* out) {
  CHECK_CHAIN(c);
  const fmc::Chain& C = c->impl;
  const fmc::InputDeck& d = C.sys.deck;
  if (dims) {
    dims[0] = (int)C.prob.size();
    for (int a = 0; a < 3; a++) dims[1 + a] = d.ngrid[a];
  }
  if (out) {
    if (plot < 0 || plot >= (int)C.prob.size()) return fail(-1, "plot index out of range");
    std::memcpy(out, C.prob[plot].data(), sizeof(double) * C.prob[plot].size());
  }
  return 0;
}

int fmc_chain_write_prob(fmc_chain* c, const char* outdir) {
  CHECK_CHAIN(c);
  if (!outdir) return fail(-1, "bad arguments");
  const fmc::Chain& C = c->impl;
  const fmc::InputDeck& d = C.sys.deck;
  if (C.prodcount <= 0) return 0;  // gcmc.f:2213: nothing is written before production
  std::vector<int> per(d.guests.size(), 0);
  for (size_t ip = 0; ip < d.plots.size(); ip++) {
    const int g = d.plots[ip].guest;
    char name[64];
    std::snprintf(name, sizeof(name), "/prob_guest%02d_prob_%02d.cube", g + 1, ++per[g]);
    std::string err;
    int rc = fmc::write_prob_cube(std::string(outdir) + name, d, C.prob[ip].data(), C.prodcount, err);
    if (rc) return fail(rc, err);
  }
  return 0;
}

int fmc_chain_pressures(fmc_chain* c, double* out) {
  CHECK_CHAIN(c);
  if (!out) return fail(-1, "bad arguments");
  const fmc::Chain& C = c->impl;
  for (size_t i = 0; i < C.gstpress.size(); i++) out[i] = C.gstpress[i];
  out[C.gstpress.size()] = C.despre;
  return 0;
}

int fmc_chain_open_outputs(fmc_chain* c, const char* outdir) {
  CHECK_CHAIN(c);
  std::string err;
  int rc = c->impl.open_outputs(outdir ? outdir : "", err);
  return rc ? fail(rc, err) : 0;
}

int fmc_chain_window_stats(fmc_chain* c, double* out) {
  CHECK_CHAIN(c);
  fmc::window_stats_out(c->impl.win, (int)c->impl.sp.size(), out);
  return 0;
}

int fmc_chain_final_stats(fmc_chain* c, double* out) {
  CHECK_CHAIN(c);
  const fmc::Chain& C = c->impl;
  fmc::final_stats((int)C.sp.size(), C.sys.deck.temp, C.chainstats.data(), C.win, C.gasmol.data(), C.gaseng.data(),
                   out);
  return 0;
}

int fmc_chain_write_report(fmc_chain* c, const char* path) {
  CHECK_CHAIN(c);
  if (!path) return fail(-1, "bad arguments");
  const fmc::Chain& C = c->impl;
  std::vector<double> cs(C.chainstats.size());
  fmc::final_stats((int)C.sp.size(), C.sys.deck.temp, C.chainstats.data(), C.win, C.gasmol.data(), C.gaseng.data(),
                   cs.data());
  std::string err;
  int rc = fmc::write_report(path, C.sys.deck, cs.data(), C.win, C.sys.deck.temp, err);
  return rc ? fail(rc, err) : 0;
}

int fmc_stats(fmc_chain* c, int iguest, double* out) {
  CHECK_CHAIN(c);
  fmc::Chain& C = c->impl;
  if (iguest < 0 || iguest >= (int)C.sp.size()) return fail(-1, "species index out of range");
  for (int i = 0; i < 5; i++) out[i] = C.chainstats[14 * iguest + 1 + i];
  out[5] = (double)C.prodcount;
  return 0;
}

int fmc_chain_profile(fmc_chain* c, int enable, double* out) {
  CHECK_CHAIN(c);
  fmc::Chain& C = c->impl;
  if (enable < 0) {
    C.passes = C.commits = C.pass_timed = 0;
    C.pass_ms = 0.0;
  }
  C.profile = enable != 0;
  if (out) {
    const fmc::HostSystem& S = C.sys;
    int nv = S.nvox[0] * S.nvox[1] * S.nvox[2];
    out[0] = (double)C.passes;
    out[1] = (double)C.commits;
    out[2] = (double)C.pass_timed;
    out[3] = C.pass_ms;
    out[4] = (double)S.K;
    out[5] = nv ? (double)C.dsys.vox_entries / nv : 0.0;
  }
  return 0;
}

int fmc_run_timed(fmc_chain* c, int nmoves, fmc_move_record* trace, float* device_ms) {
  CHECK_CHAIN(c);
  fmc::Chain& C = c->impl;
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  cudaEventRecord(a, C.st);
  int rc = fmc_run(c, nmoves, trace);
  cudaEventRecord(b, C.st);
  cudaEventSynchronize(b);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, a, b);
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  if (device_ms) *device_ms = ms;
  return rc;
}

int fmc_deck_vdw(const char* dir, int k, double* out, int* ntables) {
  if (!dir) return fail(-1, "null argument");
  fmc::InputDeck deck;
  std::string err;
  int rc = fmc::read_input_deck(dir, deck, err);
  if (rc) return fail(rc, err);
  fmc::HostSystem S;
  rc = fmc::build_host_system(deck, S, err);
  if (rc) return fail(rc, err);
  if (ntables) *ntables = S.ntables;
  if (out) {
    if (k < 1 || k > S.ntables) return fail(-1, "table index out of range");
    for (int i = 0; i <= S.mxgrid; i++) out[i] = S.vvv[(size_t)k * (S.mxgrid + 1) + i];
  }
  return 0;
}

namespace {
// Host tables of a deck: what fmc_deck_inspect and fmc_desc_inspect report.
int inspect_deck(const fmc::InputDeck& deck, int* ints, double* dbls, int* lmn, double* akk, double* erc,
                 double* charges, int* K, int* nerc, double* vvv, int* ntables) {
  fmc::HostSystem S;
  std::string err;
  int rc = fmc::build_host_system(deck, S, err);
  if (rc) return fail(rc, err);
  int nv = S.nvox[0] * S.nvox[1] * S.nvox[2];
  int natoms = S.nf;
  for (auto& g : deck.guests) natoms += g.nmols * g.nsite;
  int iv[16] = {S.cell.imcon, deck.kmax[0], deck.kmax[1], deck.kmax[2], S.K, natoms, (int)deck.guests.size(),
                S.ntypes, S.mxgrid, S.nf, 0, nv, (int)deck.plots.size(), deck.ngrid[0], deck.ngrid[1], deck.ngrid[2]};
  double dv[16] = {S.alpha, S.rcut, deck.delr, S.cell.volm, S.engunit, deck.temp, S.beta, S.drewd, S.dlrpot,
                   0, 0, 0, 0, 0, S.statvolm, 0};
  if (ints) std::memcpy(ints, iv, sizeof(iv));
  if (dbls) std::memcpy(dbls, dv, sizeof(dv));
  for (int k = 0; k < S.K; k++) {
    if (lmn) {
      lmn[3 * k] = S.kl[k];
      lmn[3 * k + 1] = S.km[k];
      lmn[3 * k + 2] = S.kn[k];
    }
    if (akk) akk[k] = S.akk[k];
  }
  if (erc)
    for (int i = 0; i <= S.mxgrid; i++) erc[i] = S.erc[i];
  if (charges)
    for (int i = 0; i < S.nf; i++) charges[i] = S.fq[i];
  if (vvv)  // rows 1..ntables, mxgrid+1 values each
    std::memcpy(vvv, S.vvv.data() + (S.mxgrid + 1), sizeof(double) * (size_t)S.ntables * (S.mxgrid + 1));
  if (K) *K = S.K;
  if (nerc) *nerc = S.mxgrid + 1;
  if (ntables) *ntables = S.ntables;
  return 0;
}
}  // namespace

int fmc_deck_inspect(const char* dir, int* ints, double* dbls, int* lmn, double* akk, double* erc, double* charges,
                     int* K, int* nerc) {
  if (!dir) return fail(-1, "null argument");
  fmc::InputDeck deck;
  std::string err;
  int rc = fmc::read_input_deck(dir, deck, err);
  if (rc) return fail(rc, err);
  return inspect_deck(deck, ints, dbls, lmn, akk, erc, charges, K, nerc, nullptr, nullptr);
}

int fmc_deck_voxels(const char* dir, double voxel_edge, int* nvox, int* off, int* atoms, long long cap,
                    long long* n_entries) {
  if (!dir || !nvox || !n_entries) return fail(-1, "null argument");
  fmc::InputDeck deck;
  fmc::HostSystem S;
  std::string err;
  int rc = fmc::read_input_deck(dir, deck, err);
  if (!rc) rc = fmc::build_host_system(deck, S, err, voxel_edge > 0.0 ? voxel_edge : 2.0);
  if (rc) return fail(rc, err);
  fmc::build_host_voxels(S);
  for (int a = 0; a < 3; a++) nvox[a] = S.nvox[a];
  *n_entries = S.vox_entries;
  if (off) std::memcpy(off, S.vox_off.data(), sizeof(int) * S.vox_off.size());
  if (atoms) {
    if (cap < S.vox_entries) return fail(-2, "atoms buffer smaller than the voxel entries");
    std::memcpy(atoms, S.vox_atoms.data(), sizeof(int) * S.vox_atoms.size());
  }
  return 0;
}

int fmc_desc_inspect(const fmc_system_desc* desc, int* ints, double* dbls, int* lmn, double* akk, double* erc,
                     double* charges, int* K, int* nerc, double* vvv, int* ntables) {
  if (!desc) return fail(-1, "null argument");
  fmc::InputDeck deck;
  std::string err;
  int rc = fmc::deck_from_desc(*desc, deck, err);
  if (rc) return fail(rc, err);
  return inspect_deck(deck, ints, dbls, lmn, akk, erc, charges, K, nerc, vvv, ntables);
}

}  // extern "C"
