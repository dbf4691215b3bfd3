// REVIVE / REVCON in the reference's formats (revive, revread: utility_pack.f:1772-1878).
#include "fmc_restart.h"

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>

namespace fmc {

namespace {

// Fortran Ew.d: 0.ddd...dE+xx, right-justified in w.
std::string fortran_e(double x, int w, int d) {
  char buf[64];
  std::string body;
  if (x == 0.0) {
    body = "0." + std::string(d, '0') + "E+00";
  } else {
    std::snprintf(buf, sizeof(buf), "%.*e", d - 1, std::fabs(x));
    std::string s(buf);  // m.mmmmE+xx
    size_t e = s.find('e');
    std::string digits = s.substr(0, 1) + s.substr(2, e - 2);
    int ex = std::atoi(s.c_str() + e + 1) + 1;
    std::snprintf(buf, sizeof(buf), "%c%02d", ex < 0 ? '-' : '+', std::abs(ex));
    body = (x < 0 ? "-0." : "0.") + digits + "E" + buf;
  }
  if ((int)body.size() < w) body = std::string(w - body.size(), ' ') + body;
  return body;
}

// Fortran Gw.d as gfortran writes it: F editing with d significant digits and four trailing
// blanks for 0.1 <= |x| < 10**d, E editing otherwise.
std::string fortran_g(double x, int w, int d) {
  char buf[64];
  if (x == 0.0) {
    std::snprintf(buf, sizeof(buf), "%*.*f", w - 4, d - 1, 0.0);
    return std::string(buf) + "    ";
  }
  std::snprintf(buf, sizeof(buf), "%.*e", d - 1, std::fabs(x));
  const char* e = std::strchr(buf, 'e');
  int k = std::atoi(e + 1) + 1;  // digits before the point of the rounded value
  if (k < 0 || k > d) return fortran_e(x, w, d);
  std::snprintf(buf, sizeof(buf), "%*.*f", w - 4, d - k, x);
  return std::string(buf) + "    ";
}

void put_record(std::ofstream& f, const void* data, uint32_t n) {
  f.write((const char*)&n, 4);
  if (n) f.write((const char*)data, n);
  f.write((const char*)&n, 4);
}

bool get_record(std::ifstream& f, std::vector<char>& out) {
  uint32_t n = 0, m = 0;
  if (!f.read((char*)&n, 4)) return false;
  out.resize(n);
  if (n && !f.read(out.data(), n)) return false;
  if (!f.read((char*)&m, 4)) return false;
  return m == n;
}

}  // namespace

Revive revive_state(const InputDeck& d, bool production, const std::vector<std::vector<double>>& guest_xyz,
                    const std::vector<double>& chainstats, const std::vector<double>& energy) {
  Revive r;
  r.production = production;
  r.chainstats = chainstats;
  r.energy = energy;
  r.natms = (int)d.fq.size();
  for (const MolLayout& m : d.mols) {
    std::vector<double> x, y, z;
    int nmol = m.nummols;
    if (m.guest >= 0) {
      const std::vector<double>& g = guest_xyz[m.guest];
      nmol = (int)(g.size() / (3 * m.numatoms));
      for (size_t i = 0; i < g.size() / 3; i++) {
        x.push_back(g[3 * i]);
        y.push_back(g[3 * i + 1]);
        z.push_back(g[3 * i + 2]);
      }
      r.natms += nmol * m.numatoms;
    } else {
      for (int i = 0; i < m.nummols * m.numatoms; i++) {
        x.push_back(d.fx[m.fw_offset + i]);
        y.push_back(d.fy[m.fw_offset + i]);
        z.push_back(d.fz[m.fw_offset + i]);
      }
    }
    r.nummols.push_back(nmol);
    r.x.push_back(x);
    r.y.push_back(y);
    r.z.push_back(z);
  }
  return r;
}

int read_revive(const std::string& path, const InputDeck& d, Revive& r, std::string& err) {
  std::ifstream f(path, std::ios::binary);
  if (!f) {
    err = "cannot open " + path;
    return -1;
  }
  const int nt = (int)d.mols.size(), ng = (int)d.guests.size();
  std::vector<char> rec;
  auto bad = [&](const char* what) {
    err = std::string("REVIVE does not match the FIELD: ") + what;
    return -2;
  };
  if (!get_record(f, rec) || rec.size() != 4) return bad("production record");
  int32_t prod;
  std::memcpy(&prod, rec.data(), 4);
  r.production = prod != 0;
  if (!get_record(f, rec) || rec.size() != 4u * nt) return bad("molecule counts");
  r.nummols.assign(nt, 0);
  std::memcpy(r.nummols.data(), rec.data(), rec.size());
  if (!get_record(f, rec) || rec.size() != 8u * (1 + 14 * ng)) return bad("chain statistics");
  r.chainstats.assign(1 + 14 * ng, 0.0);
  std::memcpy(r.chainstats.data(), rec.data(), rec.size());
  if (!get_record(f, rec) || rec.size() != 4) return bad("atom count");
  std::memcpy(&r.natms, rec.data(), 4);
  r.x.assign(nt, {});
  r.y.assign(nt, {});
  r.z.assign(nt, {});
  for (int i = 0; i < nt; i++) {
    const size_t n = (size_t)r.nummols[i] * d.mols[i].numatoms;
    if (r.nummols[i] < 0) return bad("negative molecule count");
    if (d.mols[i].guest < 0 && r.nummols[i] != d.mols[i].nummols) return bad("framework molecule count");
    for (auto* v : {&r.x[i], &r.y[i], &r.z[i]}) {
      if (!get_record(f, rec) || rec.size() != 8 * n) return bad("coordinate record length");
      v->assign(n, 0.0);
      if (n) std::memcpy(v->data(), rec.data(), rec.size());
    }
  }
  if (!get_record(f, rec) || rec.size() != 8u * ng) return bad("energies");
  r.energy.assign(ng, 0.0);
  std::memcpy(r.energy.data(), rec.data(), rec.size());
  return 0;
}

int write_revive(const std::string& path, const Revive& r, std::string& err) {
  std::ofstream f(path, std::ios::binary | std::ios::trunc);
  if (!f) {
    err = "cannot write " + path;
    return -1;
  }
  int32_t prod = r.production ? -1 : 0;
  put_record(f, &prod, 4);
  put_record(f, r.nummols.data(), 4 * (uint32_t)r.nummols.size());
  put_record(f, r.chainstats.data(), 8 * (uint32_t)r.chainstats.size());
  int32_t natms = r.natms;
  put_record(f, &natms, 4);
  for (size_t i = 0; i < r.x.size(); i++) {
    put_record(f, r.x[i].data(), 8 * (uint32_t)r.x[i].size());
    put_record(f, r.y[i].data(), 8 * (uint32_t)r.y[i].size());
    put_record(f, r.z[i].data(), 8 * (uint32_t)r.z[i].size());
  }
  put_record(f, r.energy.data(), 8 * (uint32_t)r.energy.size());
  if (!f) {
    err = "write failed: " + path;
    return -1;
  }
  return 0;
}

int write_revcon(const std::string& path, const InputDeck& d, const Revive& r, double eng, std::string& err) {
  std::ofstream f(path, std::ios::trunc);
  if (!f) {
    err = "cannot write " + path;
    return -1;
  }
  char buf[128];
  std::string title = d.title.substr(0, 80);
  title.resize(80, ' ');
  f << title << '\n';
  std::snprintf(buf, sizeof(buf), "%10d%10d", 0, d.imcon);
  f << buf << fortran_e(eng, 20, 10) << '\n';
  if (d.imcon > 0)
    for (int row = 0; row < 3; row++) {
      for (int j = 0; j < 3; j++) {
        std::snprintf(buf, sizeof(buf), "%20.12f", d.cell[3 * row + j]);
        f << buf;
      }
      f << '\n';
    }
  int idx = 0;
  auto atom = [&](const std::string& name, double x, double y, double z) {
    std::string n = name.substr(0, 8);
    n.resize(8, ' ');
    std::snprintf(buf, sizeof(buf), "%10d", ++idx);
    f << n << buf << '\n' << fortran_g(x, 20, 10) << fortran_g(y, 20, 10) << fortran_g(z, 20, 10) << '\n';
  };
  // condensed order: every guest species first (condense, utility_pack.f:3325-3423), then the
  // framework molecule types in FIELD order
  for (size_t g = 0; g < d.guests.size(); g++)
    for (size_t i = 0; i < d.mols.size(); i++)
      if (d.mols[i].guest == (int)g) {
        const GuestSpecies& G = d.guests[g];
        for (size_t s = 0; s < r.x[i].size(); s++) atom(G.site_name[s % G.nsite], r.x[i][s], r.y[i][s], r.z[i][s]);
      }
  for (size_t i = 0; i < d.mols.size(); i++)
    if (d.mols[i].guest < 0)
      for (size_t s = 0; s < r.x[i].size(); s++)
        atom(d.fname[d.mols[i].fw_offset + s], r.x[i][s], r.y[i][s], r.z[i][s]);
  if (!f) {
    err = "write failed: " + path;
    return -1;
  }
  return 0;
}

std::vector<std::vector<double>> revive_guest_xyz(const InputDeck& d, const Revive& r) {
  std::vector<std::vector<double>> out(d.guests.size());
  for (size_t i = 0; i < d.mols.size(); i++) {
    int g = d.mols[i].guest;
    if (g < 0) continue;
    std::vector<double>& v = out[g];
    v.resize(3 * r.x[i].size());
    for (size_t s = 0; s < r.x[i].size(); s++) {
      v[3 * s] = r.x[i][s];
      v[3 * s + 1] = r.y[i][s];
      v[3 * s + 2] = r.z[i][s];
    }
  }
  return out;
}

}  // namespace fmc
