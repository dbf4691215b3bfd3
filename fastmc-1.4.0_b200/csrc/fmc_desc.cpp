// Systems handed over as arrays (fmc_system_desc) instead of deck files, and decks read into
// such descriptors.  The descriptor holds what the reference's module arrays hold once its
// readers have run (utility_pack.f:8-68, vdw_module.f:19-24): coordinates, charges and 1-based
// types of the framework, the guest templates already centred on their mass centres
// (readinputs.f:246-268), the molecules present, the vdW pair lines with energies in internal
// units, and the CONTROL values.  Both routes end in the same InputDeck, so a chain created from
// a descriptor builds the same tables and runs the same trajectory as one opened from the files
// the descriptor was read from.
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "../../include/fastmc_b200.h"
#include "fmc_desc.h"

namespace fmc {

namespace {

std::string pad8(const std::string& s) {
  std::string t = s.substr(0, 8);
  t.resize(8, ' ');
  return t;
}

// Storage behind a descriptor that fmc_deck_describe fills (released by fmc_desc_free).
struct DescStore {
  InputDeck deck;
  std::vector<std::string> type_names;
  std::vector<const char*> type_ptrs;
  std::vector<std::vector<const char*>> site_ptrs;
  std::vector<std::string> guest_names;
  std::vector<double> fw_xyz;
  std::vector<fmc_guest_desc> guests;
  std::vector<fmc_vdw_desc> vdw;
};

}  // namespace

int deck_from_desc(const fmc_system_desc& D, InputDeck& d, std::string& err) {
  d = InputDeck();
  const int nt = D.ntypes, nf = D.nframework, ng = D.nguest;
  if (nt < 1 || nf < 0 || ng < 1 || ng > kMaxGuestTypes || D.nvdw < 0) {
    err = "descriptor counts out of range (types >= 1, species 1-" + std::to_string(kMaxGuestTypes) + ")";
    return -1;
  }
  if (nf > 0 && (!D.fw_xyz || !D.fw_charge || !D.fw_type)) {
    err = "framework arrays missing";
    return -1;
  }
  if (!D.guests || (D.nvdw > 0 && !D.vdw)) {
    err = "guest or vdW arrays missing";
    return -1;
  }
  d.imcon = D.imcon;
  std::memcpy(d.cell, D.cell, sizeof(d.cell));
  d.alpha = D.alpha;
  for (int a = 0; a < 3; a++) d.kmax[a] = D.kmax[a];
  d.rcut = D.rcut;
  d.rvdw = D.rvdw;
  d.delr = D.delr;
  d.engunit = D.engunit > 0.0 ? D.engunit : 1.0;
  d.maxguest = D.max_guest_atoms > 0 ? D.max_guest_atoms : 3000;
  for (int t = 0; t < nt; t++) {
    char buf[16];
    std::snprintf(buf, sizeof(buf), "T%d", t + 1);
    d.types.push_back(pad8(D.type_names && D.type_names[t] ? std::string(D.type_names[t]) : std::string(buf)));
  }
  for (int g = 0; g < ng; g++) {
    const fmc_guest_desc& G = D.guests[g];
    const int ns = G.nsite;
    if (ns < 1 || ns > 50 || !G.mass || !G.charge || !G.tx || !G.ty || !G.tz || !G.type ||
        (G.nmols > 0 && !G.xyz) || G.nmols < 0) {
      err = "guest species " + std::to_string(g) + ": sites outside 1-50 or arrays missing";
      return -1;
    }
    GuestSpecies s;
    std::string name = G.name ? std::string(G.name) : std::string("guest");
    name.resize(40, ' ');
    s.name = name;
    s.nsite = ns;
    for (int i = 0; i < ns; i++) {
      if (G.type[i] < 1 || G.type[i] > nt) {
        err = "guest site of an unknown type";
        return 4;
      }
      s.site_name.push_back(G.site_name && G.site_name[i] ? pad8(G.site_name[i]) : d.types[G.type[i] - 1]);
      s.mass.push_back(G.mass[i]);
      s.charge.push_back(G.charge[i]);
      s.tx.push_back(G.tx[i]);
      s.ty.push_back(G.ty[i]);
      s.tz.push_back(G.tz[i]);
      s.type.push_back(G.type[i]);
    }
    s.nmols = G.nmols;
    s.xyz.assign(G.xyz, G.xyz + 3 * (size_t)G.nmols * ns);
    d.guests.push_back(s);
    d.mols.push_back({g, 0, G.nmols, ns});
    d.press.push_back(G.pressure_pa);
    std::array<double, 9> mf;
    for (int k = 0; k < 9; k++) mf[k] = G.move_freq[k];
    d.movefreq.push_back(mf);
    d.disp_ratio.push_back(G.disp_ratio > 0.0 ? G.disp_ratio : 0.5);
    d.tran_ratio.push_back(G.tran_ratio > 0.0 ? G.tran_ratio : 0.5);
  }
  d.adspres.assign(ng, 0.0);
  d.adsguen.assign(ng, 0.0);
  for (int i = 0; i < nf; i++) {
    const int t = D.fw_type[i];
    if (t < 1 || t > nt) {
      err = "framework atom of an unknown type";
      return 4;
    }
    d.fx.push_back(D.fw_xyz[3 * i]);
    d.fy.push_back(D.fw_xyz[3 * i + 1]);
    d.fz.push_back(D.fw_xyz[3 * i + 2]);
    d.fq.push_back(D.fw_charge[i]);
    d.ftype.push_back(t);
    d.ffrz.push_back(1);
    d.fname.push_back(d.types[t - 1]);
    d.fmass.push_back(D.fw_mass ? D.fw_mass[i] : 0.0);
  }
  if (nf > 0) d.mols.push_back({-1, 0, 1, nf});
  // vdW pair lines: loc8 key of the pair -> line (define_van_der_waals)
  d.ntpvdw = D.nvdw;
  d.ltpvdw.assign(D.nvdw + 1, -1);
  d.prmvdw.assign(D.nvdw + 1, {0, 0, 0, 0, 0});
  d.lstvdw.assign(nt * (nt + 1) / 2 + 1, 0);
  for (int l = 0; l < D.nvdw; l++) {
    const fmc_vdw_desc& V = D.vdw[l];
    if (V.type_i < 1 || V.type_i > nt || V.type_j < 1 || V.type_j > nt || V.form < 1 || V.form > 9) {
      err = "vdW line " + std::to_string(l) + ": unknown type or form";
      return 4;
    }
    const int hi = std::max(V.type_i, V.type_j), lo = std::min(V.type_i, V.type_j);
    d.lstvdw[hi * (hi - 1) / 2 + lo] = l + 1;
    d.ltpvdw[l + 1] = V.form;
    for (int k = 0; k < 5; k++) d.prmvdw[l + 1][k] = V.prm[k];
  }
  d.temp = D.temperature;
  d.eqsteps = D.eq_steps;
  d.mcsteps = D.prod_steps;
  d.nwind = D.averaging_window > 0 ? D.averaging_window : 100000;
  d.laccsample = D.acceptance_sampling != 0;
  d.rota_ratio = D.rota_ratio > 0.0 ? D.rota_ratio : 0.5;
  d.title = "system created from caller arrays";
  return finish_deck_from_arrays(d, err);
}

int describe_deck(const std::string& dir, fmc_system_desc& D, std::string& err) {
  auto st = std::make_unique<DescStore>();
  int rc = read_input_deck(dir, st->deck, err);
  if (rc) return rc;
  const InputDeck& d = st->deck;
  for (int f : d.ffrz)
    if (f == 0) {
      err = "framework atoms must be frozen (rigid framework)";
      return -6;
    }
  std::memset(&D, 0, sizeof(D));
  D.imcon = d.imcon;
  std::memcpy(D.cell, d.cell, sizeof(D.cell));
  D.alpha = d.alpha;
  for (int a = 0; a < 3; a++) D.kmax[a] = d.kmax[a];
  D.rcut = d.rcut;
  D.rvdw = d.rvdw;
  D.delr = d.delr;
  D.engunit = d.engunit;
  D.ntypes = (int)d.types.size();
  for (const std::string& t : d.types) st->type_ptrs.push_back(t.c_str());
  D.type_names = st->type_ptrs.data();
  D.nframework = (int)d.fq.size();
  for (int i = 0; i < D.nframework; i++) {
    st->fw_xyz.push_back(d.fx[i]);
    st->fw_xyz.push_back(d.fy[i]);
    st->fw_xyz.push_back(d.fz[i]);
  }
  D.fw_xyz = st->fw_xyz.data();
  D.fw_charge = d.fq.data();
  D.fw_type = d.ftype.data();
  D.fw_mass = d.fmass.data();
  const int ng = (int)d.guests.size();
  st->site_ptrs.resize(ng);
  for (int g = 0; g < ng; g++) {
    const GuestSpecies& s = d.guests[g];
    for (const std::string& n : s.site_name) st->site_ptrs[g].push_back(n.c_str());
    fmc_guest_desc G;
    std::memset(&G, 0, sizeof(G));
    G.name = s.name.c_str();
    G.nsite = s.nsite;
    G.site_name = st->site_ptrs[g].data();
    G.mass = s.mass.data();
    G.charge = s.charge.data();
    G.tx = s.tx.data();
    G.ty = s.ty.data();
    G.tz = s.tz.data();
    G.type = s.type.data();
    G.nmols = s.nmols;
    G.xyz = s.xyz.empty() ? nullptr : s.xyz.data();
    G.pressure_pa = d.press[g];
    for (int k = 0; k < 9; k++) G.move_freq[k] = d.movefreq[g][k];
    G.disp_ratio = d.disp_ratio[g];
    G.tran_ratio = d.tran_ratio[g];
    st->guests.push_back(G);
  }
  D.nguest = ng;
  D.guests = st->guests.data();
  // every pair line the deck names, in FIELD order (each referenced by the loc8 key of its pair)
  const int nt = D.ntypes;
  for (int l = 1; l <= d.ntpvdw; l++) {
    for (int hi = 1; hi <= nt; hi++)
      for (int lo = 1; lo <= hi; lo++)
        if (d.lstvdw[hi * (hi - 1) / 2 + lo] == l) {
          fmc_vdw_desc V;
          V.type_i = hi;
          V.type_j = lo;
          V.form = d.ltpvdw[l];
          for (int k = 0; k < 5; k++) V.prm[k] = d.prmvdw[l][k];
          st->vdw.push_back(V);
        }
  }
  if ((int)st->vdw.size() != d.ntpvdw) {
    err = "a vdW line of the deck names a pair another line redefines";
    return -1;
  }
  D.nvdw = (int)st->vdw.size();
  D.vdw = st->vdw.data();
  D.temperature = d.temp;
  D.eq_steps = d.eqsteps;
  D.prod_steps = d.mcsteps;
  D.max_guest_atoms = d.maxguest;
  D.averaging_window = d.nwind;
  D.acceptance_sampling = d.laccsample ? 1 : 0;
  D.rota_ratio = d.rota_ratio;
  D.owner = st.release();
  return 0;
}

void free_desc(fmc_system_desc& D) {
  delete static_cast<DescStore*>(D.owner);
  std::memset(&D, 0, sizeof(D));
}

}  // namespace fmc
