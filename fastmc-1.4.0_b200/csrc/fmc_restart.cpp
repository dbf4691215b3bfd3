// REVIVE / REVCON in the reference's formats (revive, revread: utility_pack.f:1772-1878).
#include "fmc_restart.h"

#include <dirent.h>
#include <sys/stat.h>

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

int atomic_number(double mass) {
  // mass windows -> atomic number, the same windows as the reference's atmnumber so that the
  // cube files label framework atoms alike (first matching window wins; 0 when none matches)
  struct Win {
    double lo, hi;
    int z;
  };
  static const Win win[] = {
      {0, 1.5, 1}, {3.9, 4.5, 2}, {6.5, 7.1, 3}, {8.9, 9.5, 4}, {10.5, 11.1, 5}, {11.9, 12.5, 6}, {13.9, 14.5, 7},
      {15.5, 16.1, 8}, {18.5, 19.1, 9}, {19.9, 20.5, 10}, {22.5, 23.1, 11}, {23.9, 24.5, 12}, {26.5, 27.1, 13},
      {27.9, 28.5, 14}, {30.5, 31.1, 15}, {31.9, 32.5, 16}, {34.9, 36.1, 17}, {39.5, 39.9999, 18},
      {38.9, 39.4, 19}, {40, 40.5, 20}, {44.5, 45.1, 21}, {47.5, 48.1, 22}, {50.5, 51.1, 23}, {51.5, 52.1, 24},
      {54.5, 55.1, 25}, {55.5, 56.1, 26}, {58.76, 59.1, 27}, {58.5, 59.75, 28}, {62.9, 64.1, 29}, {64.9, 66.1, 30},
      {69.5, 70.1, 31}, {72.5, 73.1, 32}, {74.5, 75.1, 33}, {78.5, 79.1, 34}, {79.5, 80.1, 35}, {83.5, 84.1, 36},
      {84.9, 86.1, 37}, {87.5, 88.1, 38}, {88.5, 89.1, 39}, {90.9, 91.5, 40}, {92.5, 93.1, 41}, {95.5, 96.1, 42},
      {97.9, 98.1, 43}, {109.9, 101.5, 44}, {102.5, 103.1, 45}, {105.9, 106.5, 46}, {107.5, 108.1, 47},
      {111.9, 112.5, 48}, {114.5, 115.1, 49}, {118.5, 119.1, 50}, {121.5, 122.1, 51}, {127.5, 128.1, 52},
      {126.5, 127.1, 53}, {130.9, 131.5, 54}, {132.5, 133.1, 55}, {136.9, 137.5, 56}, {138.5, 139.1, 57},
      {139.9, 140.5, 58}, {140.6, 141.1, 59}, {144, 144.5, 60}, {144.9, 145.1, 61}, {150, 150.6, 62},
      {151.5, 152.1, 63}, {156.9, 157.5, 64}, {158.5, 159.1, 65}, {162, 163.1, 66}, {164.5, 165.1, 67},
      {166.5, 167.9, 68}, {168, 169.1, 69}, {172.9, 173.5, 70}, {174, 175.1, 71}, {178, 179.1, 72},
      {180, 181.1, 73}, {183, 184.1, 74}, {185.9, 186.5, 75}, {189.9, 190.5, 76}, {191.9, 192.5, 77},
      {194.9, 195.5, 78}, {196.5, 197.1, 79}, {200, 201.1, 80}, {203.9, 204.6, 81}, {206.9, 207.6, 82},
      {208.5, 209.1, 83}, {209.9, 210.1, 85}, {221.9, 222.1, 86}, {222.9, 223.1, 87}, {225.9, 226.1, 88},
      {226.9, 227.1, 89}, {231.9, 232.1, 90}, {230.9, 231.1, 91}, {237.9, 238.1, 92}, {243.9, 244.1, 94},
      {242.9, 243.1, 95}, {246.9, 247.1, 96}, {250.9, 251.1, 98}, {251.9, 252.1, 99}, {256.9, 257.1, 100},
      {257.9, 258.1, 101}, {258.9, 259.1, 102}, {261.9, 262.1, 103}, {266.9, 267.1, 104}, {267.9, 268.1, 105},
      {270.9, 271.1, 106}, {269.9, 270.1, 107}, {268.9, 269.1, 108}, {277.9, 278.1, 109}, {280.9, 281.1, 110},
      {284.9, 285.1, 112}, {285.9, 286.1, 113}, {288.9, 289.1, 114}, {292.9, 293.1, 116}, {293.9, 294.1, 117}};
  for (const Win& v : win)
    if (mass >= v.lo && mass <= v.hi) return v.z;
  return 0;
}

int write_prob_cube(const std::string& path, const InputDeck& d, const double* grid, long long steps,
                    std::string& err) {
  std::ofstream f(path, std::ios::trunc);
  if (!f) {
    err = "cannot write " + path;
    return -1;
  }
  const double a2b = 1.889725989;  // Angstrom -> Bohr (utility_pack.f:82)
  double c[9];
  for (int i = 0; i < 9; i++) c[i] = d.cell[i] * a2b;
  const int na = d.ngrid[0], nb = d.ngrid[1], nc = d.ngrid[2];
  // volume of one grid cell (writeprob), in Bohr^3
  const double vol = (c[1] * c[5] - c[2] * c[4]) / (na * nb) * c[6] / nc +
                     (c[2] * c[3] - c[0] * c[5]) / (na * nb) * c[7] / nc +
                     (c[0] * c[4] - c[1] * c[3]) / (na * nb) * c[8] / nc;
  char buf[160];
  // the second line keeps the blanks the reference's fixed-form continuation puts in it
  f << "probability cube file\n" << "outer loop a, middle loop     b, inner loop c\n";
  const int nf = (int)d.fq.size();
  std::snprintf(buf, sizeof(buf), "%6d%12.6f%12.6f%12.6f\n", nf, 0.0, 0.0, 0.0);
  f << buf;
  const int n[3] = {na, nb, nc};
  for (int a = 0; a < 3; a++) {
    std::snprintf(buf, sizeof(buf), "%6d%12.6f%12.6f%12.6f\n", n[a], c[3 * a] / n[a], c[3 * a + 1] / n[a],
                  c[3 * a + 2] / n[a]);
    f << buf;
  }
  for (int i = 0; i < nf; i++) {
    std::snprintf(buf, sizeof(buf), "%6d%12.6f%12.6f%12.6f%12.6f\n", atomic_number(d.fmass[i]), 0.0, d.fx[i] * a2b,
                  d.fy[i] * a2b, d.fz[i] * a2b);
    f << buf;
  }
  const long long total = (long long)na * nb * nc;
  int ip = 0;
  for (long long j = 1; j <= total; j++) {
    ip++;
    f << fortran_e(grid[j - 1] / vol / (double)steps, 15, 6);
    if (j % nc == 0 || ip == 6) {
      f << '\n';
      ip = 0;
    }
  }
  if (!f) {
    err = "write failed: " + path;
    return -1;
  }
  return 0;
}

void final_stats(int ng, double temp, const double* chainstats, const WindowStats& W, const double* gasmol,
                 const double* gaseng, double* out) {
  const int windn = 5;  // gcmc.f:119
  std::vector<double> cs(chainstats, chainstats + 1 + 14 * ng);
  WindowStats V = W;
  int avcount = V.avcount;
  const double weight = cs[0];
  if (weight > 0) {
    for (int i = 0; i < ng; i++) {
      const int is = 1 + 14 * i;
      if (weight <= kSampleCap) {
        const long long nw = (long long)weight / windn;
        avcount = windn;
        double sum[8] = {0}, var[8] = {0};
        for (int x = 1; x <= windn; x++) {
          const size_t y = (size_t)i * kSampleCap + (size_t)(x - 1) * nw;
          const size_t cap = (size_t)ng * kSampleCap + 1;
          double an = 0, e = 0, en = 0, n2 = 0, e2 = 0;
          for (size_t k = y; k <= y + (size_t)nw; k++) {
            const double m = (gasmol && k < cap) ? gasmol[k] : 0.0, g = (gaseng && k < cap) ? gaseng[k] : 0.0;
            an += m;
            e += g;
            en += m * g;
            n2 += m * m;
            e2 += g * g;
          }
          double avg[7];
          avg[0] = an / nw;
          avg[1] = e / nw;
          avg[2] = en / nw;
          avg[3] = n2 / nw;
          avg[4] = e2 / nw;
          avg[5] = calc_qst(avg[4], avg[1], avg[0], avg[3], avg[2], temp);
          avg[6] = calc_cv(avg[4], avg[1], avg[0], avg[3], avg[2], temp);
          for (int z = 0; z < 7; z++) {
            const double delta = avg[z] - sum[z];
            sum[z] = sum[z] + delta / x;
            var[z] = var[z] + delta * (avg[z] - sum[z]);
          }
        }
        for (int z = 0; z < 6; z++) cs[is + z] = sum[z];
        for (int z = 0; z < 8; z++) V.var[i][z] = z < 7 ? var[z] : 0.0;
      }
      for (int z = 0; z < 8; z++) cs[is + 6 + z] = std::sqrt(V.var[i][z] / avcount);
    }
  }
  std::memcpy(out, cs.data(), sizeof(double) * cs.size());
}

void window_stats_out(const WindowStats& W, int ng, double* out) {
  out[0] = W.avcount;
  out[1] = W.rollcount;
  double* o = out + 2;
  for (int i = 0; i < ng; i++)
    for (int k = 0; k < 8; k++) {
      o[8 * i + k] = W.sum[i][k];
      o[8 * ng + 8 * i + k] = W.var[i][k];
      o[16 * ng + 8 * i + k] = W.avg[i][k];
    }
  for (int i = 0; i < ng; i++)
    for (int j = 0; j < ng; j++) o[24 * ng + i * ng + j] = W.seltot[i][j];
}

int write_report(const std::string& path, const InputDeck& d, const double* cs, const WindowStats& W, double temp,
                 std::string& err) {
  std::ofstream f(path, std::ios::trunc);
  if (!f) {
    err = "cannot write " + path;
    return -1;
  }
  char buf[256];
  const std::string stars(75, '*');
  f << "\n" << stars << "\n   Data reported from node   0\n" << stars << "\n\n";
  // one record per value, a blank record after each block (the formats of gcmc.f:2095-2108)
  auto row = [&](const char* label, double v) {
    std::snprintf(buf, sizeof(buf), "     %60s%20.9f\n", label, v);
    f << buf;
  };
  const int ng = (int)d.guests.size();
  for (int i = 0; i < ng; i++) {
    const double* c = cs + 1 + 14 * i;
    std::string name = d.guests[i].name.substr(0, 40);
    name.resize(40, ' ');
    std::snprintf(buf, sizeof(buf), "     guest %2d: %s\n\n", i + 1, name.c_str());
    f << buf;
    row("<N>: ", c[0]);
    row("<E>: ", c[1]);
    row("<E*N>: ", c[2]);
    row("<N*N>: ", c[3]);
    row("<E*E>: ", c[4]);
    std::snprintf(buf, sizeof(buf), "     %60s%20lld\n", "Multiplier: ", (long long)cs[0]);
    f << buf;
    row("Isosteric heat of adsorption (kcal/mol): ", calc_qst(c[4], c[1], c[0], c[3], c[2], temp));
    row("Isosteric heat error: ", c[11]);
    row("Heat capacity, Cv (kcal/mol/K): ", calc_cv(c[4], c[1], c[0], c[3], c[2], temp));
    row("Heat capacity error: ", c[12]);
    f << "\n";
  }
  if (ng > 1)
    for (int i = 0; i < ng; i++)
      for (int j = 0; j < i; j++) {
        std::snprintf(buf, sizeof(buf), "     guest %2d over guest %2d\n\n", j + 1, i + 1);
        f << buf;
        row("<S>: ", W.seltot[i][j]);
        f << "\n";
      }
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

int choose_branch(const std::string& workdir, int idnode, BranchChoice& out, std::string& err) {
  out = BranchChoice();
  if (idnode < 0 || idnode > 98) {
    err = "node index outside 0-98 (branch directories are named branch01-branch99)";
    return -1;
  }
  // `ls | grep -c branch`: every listed name (not the hidden ones) that contains "branch"
  if (DIR* dp = opendir(workdir.c_str())) {
    while (dirent* e = readdir(dp))
      if (e->d_name[0] != '.' && std::strstr(e->d_name, "branch")) out.prevnodes++;
    closedir(dp);
  }
  auto branch = [&](int n) {
    char b[16];
    std::snprintf(b, sizeof(b), "branch%02d", n);
    return workdir + "/" + b;
  };
  out.outdir = branch(idnode + 1);
  if (out.prevnodes == 0) return 0;
  const std::string local = idnode + 1 > out.prevnodes ? branch((idnode + 1) % out.prevnodes + 1) : out.outdir;
  struct stat sb;
  if (stat((local + "/REVIVE").c_str(), &sb) == 0 && S_ISREG(sb.st_mode)) out.revive = local + "/REVIVE";
  return 0;
}

}  // namespace fmc
