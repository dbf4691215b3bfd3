// Reader of FastMC's CONTROL / FIELD / CONFIG decks.  The record semantics are the
// reference's DL_POLY parser (parse_module.f): 150-character blank-padded records,
// substring keyword tests on lower-cased, left-stripped records, and numbers taken from the
// front of the record by intstr/dblstr (which consume what they read).  They are kept exactly
// because the directive order and number scanning decide what a deck means.
#include "fmc_inputs.h"

#include <algorithm>
#include <charconv>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <string_view>

namespace fmc {
namespace {

constexpr int kRecLen = 150;

struct InputError {
  int code;
  std::string msg;
};
[[noreturn]] void raise(int code, const std::string& msg) { throw InputError{code, msg}; }

class Record {
 public:
  char c[kRecLen];
  void set(const char* s, size_t n) {
    const int m = n < (size_t)kRecLen ? (int)n : kRecLen;
    for (int i = 0; i < m; i++) {
      const char ch = s[i];
      c[i] = (ch == '\t' || ch == '\r') ? ' ' : ch;
    }
    std::memset(c + m, ' ', kRecLen - m);
  }
  // lowcase (parse_module.f:331): only the first n characters
  void lower(int n = kRecLen) {
    for (int i = 0; i < n; i++)
      if (c[i] >= 'A' && c[i] <= 'Z') c[i] = char(c[i] - 'A' + 'a');
  }
  // strip (parse_module.f:290): drop leading blanks
  void strip() {
    int k = 0;
    while (k < kRecLen && c[k] == ' ') k++;
    if (k == 0) return;
    std::memmove(c, c + k, kRecLen - k);
    std::memset(c + kRecLen - k, ' ', k);
  }
  bool blank_or_comment() const { return c[0] == '#' || c[0] == ' '; }
  // findstring (parse_module.f:449): substring anywhere in the record
  bool has(const char* s) const {
    size_t n = std::strlen(s);
    for (size_t h = 0; h + n <= (size_t)kRecLen; h++)
      if (std::memcmp(c + h, s, n) == 0) return true;
    return false;
  }
  // Drops the first `lst` characters (parse_module.f:158-163 shift of the consumed text).
  void consume(int lst) {
    if (lst <= 1) return;
    int keep = kRecLen - lst + 1;
    std::memmove(c, c + lst - 1, keep);
    std::memset(c + keep, ' ', kRecLen - keep);
  }
  // intstr (parse_module.f:96): first digit run, negative if preceded by '-'
  int take_int() {
    int lst = 0;
    int v = scan_int(c, kRecLen, &lst);
    consume(lst);
    return v;
  }
  // dblstr (parse_module.f:171): digits accumulated left to right, fraction digits scaled
  // by successive divisions of 1 by 10, optional d/e exponent.
  double take_double() {
    int lst = 0, idum = 0, iexp = 0;
    double sn = 1.0, ten = 10.0, one = 1.0, v = 0.0;
    char prev = '+';
    bool start = false, ldot = false, fin = false;
    while (lst < kRecLen && !fin) {
      char ch = c[lst++];
      bool digit = ch >= '0' && ch <= '9';
      bool flag = digit || ch == '.';
      if (digit) v = ten * v + one * (double)(ch - '0');
      if (ch == '.') {
        ten = 1.0;
        ldot = true;
      }
      if (flag) start = true;
      if (flag && prev == '-') sn = -1.0;
      if (ldot) one = one / 10.0;
      prev = ch == 'D' ? 'd' : (ch == 'E' ? 'e' : ch);
      if (start) {
        if (prev == 'd' || prev == 'e') {
          iexp = scan_int(c + lst, kRecLen - lst, &idum);
          fin = true;
        }
        if (!flag) fin = true;
      }
    }
    v = sn * v * ipow10(iexp);
    consume(lst + idum);
    return v;
  }
  // getword (parse_module.f:547): next blank-delimited word, at most len1 characters,
  // returned blank-padded to 8 characters.
  // The reference shifts the record one character per character examined; the shift is done
  // once here, by the number examined.
  std::string take_word(int len1) {
    char w[kRecLen];
    int nw = 0, i = 0;
    bool fin = false;
    while (!fin && i < kRecLen) {
      const char ch = c[i++];
      if (ch == ' ') {
        if (nw) fin = true;
      } else {
        w[nw++] = ch;
        if (nw == len1) fin = true;
      }
    }
    std::memmove(c, c + i, kRecLen - i);
    std::memset(c + kRecLen - i, ' ', i);
    std::string out(w, nw);
    out.resize(8, ' ');
    return out;
  }

 private:
  static int scan_int(const char* w, int len, int* lst_out) {
    int isn = 1, lst = 0, v = 0;
    char prev = '+';
    bool seen = false, fin = false;
    while (lst < len && !fin) {
      char ch = w[lst++];
      bool digit = ch >= '0' && ch <= '9';
      if (digit) {
        v = 10 * v + (ch - '0');
        seen = true;
      }
      if (seen && !digit) fin = true;
      if (digit && prev == '-') isn = -1;
      prev = ch;
    }
    *lst_out = lst;
    return isn * v;
  }
  // real(8)**integer as compiled by gfortran (binary powering, reciprocal for negatives)
  static double ipow10(int m) {
    unsigned n = m < 0 ? -(unsigned)m : (unsigned)m;
    double x = 10.0, y = (n & 1) ? x : 1.0;
    while (n >>= 1) {
      x = x * x;
      if (n & 1) y = y * x;
    }
    return m < 0 ? 1.0 / y : y;
  }
};

// A file read whole, served a line at a time (lines as std::getline splits them: at '\n', the
// last one counted only when it holds characters).
class Deck {
 public:
  Deck(const std::string& path, int eof_code, const char* eof_msg) : code_(eof_code), msg_(eof_msg) {
    std::ifstream f(path, std::ios::binary);
    if (!f) raise(code_, std::string("cannot open ") + path);
    f.seekg(0, std::ios::end);
    const std::streamoff n = f.tellg();
    f.seekg(0, std::ios::beg);
    buf_.resize(n > 0 ? (size_t)n : 0);
    if (n > 0 && !f.read(&buf_[0], n)) raise(code_, std::string("cannot read ") + path);
    size_t at = 0;
    while (at < buf_.size()) {
      const void* nl = std::memchr(buf_.data() + at, '\n', buf_.size() - at);
      const size_t end = nl ? (size_t)((const char*)nl - buf_.data()) : buf_.size();
      lines_.push_back({at, end - at});
      at = end + 1;
    }
  }
  Record next() {
    if (pos_ >= lines_.size()) raise(code_, msg_);
    Record r;
    const Line& l = lines_[pos_++];
    r.set(buf_.data() + l.at, l.len);
    return r;
  }
  std::string_view raw() {
    if (pos_ >= lines_.size()) raise(55, "end of CONFIG file encountered");
    const Line& l = lines_[pos_++];
    return std::string_view(buf_.data() + l.at, l.len);
  }

 private:
  struct Line {
    size_t at, len;
  };
  std::string buf_;
  std::vector<Line> lines_;
  size_t pos_ = 0;
  int code_;
  std::string msg_;
};

// Perpendicular widths and volume of a cell (dcell, utility_pack.f:1351-1415)
void cell_props(const double* a, double* b) {
  double axb[3] = {a[1] * a[5] - a[2] * a[4], a[2] * a[3] - a[0] * a[5], a[0] * a[4] - a[1] * a[3]};
  double bxc[3] = {a[4] * a[8] - a[5] * a[7], a[5] * a[6] - a[3] * a[8], a[3] * a[7] - a[4] * a[6]};
  double cxa[3] = {a[7] * a[2] - a[1] * a[8], a[0] * a[8] - a[2] * a[6], a[1] * a[6] - a[0] * a[7]};
  b[0] = std::sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
  b[1] = std::sqrt(a[3] * a[3] + a[4] * a[4] + a[5] * a[5]);
  b[2] = std::sqrt(a[6] * a[6] + a[7] * a[7] + a[8] * a[8]);
  b[9] = std::fabs(a[0] * bxc[0] + a[1] * bxc[1] + a[2] * bxc[2]);
  b[6] = b[9] / std::sqrt(bxc[0] * bxc[0] + bxc[1] * bxc[1] + bxc[2] * bxc[2]);
  b[7] = b[9] / std::sqrt(cxa[0] * cxa[0] + cxa[1] * cxa[1] + cxa[2] * cxa[2]);
  b[8] = b[9] / std::sqrt(axb[0] * axb[0] + axb[1] * axb[1] + axb[2] * axb[2]);
}

double half_width(const InputDeck& d, const double* cp) {
  double w = std::min(cp[6], std::min(cp[7], cp[8])) / 2.0;
  if (d.imcon == 4) w = std::sqrt(3.0) * d.cell[0] / 4.0;
  if (d.imcon == 5) w = d.cell[0] / 2.0;
  if (d.imcon == 6) w = std::min(cp[6], cp[7]) / 2.0;
  return w;
}

double volume_of(int imcon, const double* cp) {
  if (imcon == 0) return 0.0;
  if (imcon == 4 || imcon == 5 || imcon == 7) return 0.5 * cp[9];
  return cp[9];
}

// ---------------------------------------------------------------- pre-scan (initscan)
struct Scan {
  int mxatyp = 0;
  int nguest_control = 0;
  bool lewald = false;
};

void prescan(const std::string& dir, InputDeck& d, Scan& s) {
  {
    Deck f(dir + "/FIELD", 52, "end of FIELD file encountered");
    f.next();
    std::vector<std::string> names;
    for (;;) {
      Record r = f.next();
      r.lower();
      r.strip();
      if (r.blank_or_comment()) continue;
      if (r.has("molecu")) {
        int nmol_types = r.take_int(), nummls = 0;
        for (int n = 0; n < nmol_types; n++) {
          for (;;) {
            Record m = f.next();
            m.lower();
            m.strip();
            if (m.blank_or_comment()) continue;
            if (m.has("nummol")) {
              nummls = m.take_int();
            } else if (m.has("atoms")) {
              int numsit = m.take_int(), ksite = 0;
              for (int i = 0; i < numsit; i++) {
                if (ksite >= numsit) continue;
                Record a = f.next();
                std::string name = a.take_word(8);
                a.take_double();
                a.take_double();
                int nrept = a.take_int();
                ksite += nrept == 0 ? 1 : nrept;
                if (std::find(names.begin(), names.end(), name) == names.end()) names.push_back(name);
              }
            } else if (m.has("finish")) {
              break;
            }
          }
          (void)nummls;
        }
      } else if (r.has("vdw")) {
        d.ntpvdw = r.take_int();
      } else if (r.has("close")) {
        break;
      }
    }
    s.mxatyp = (int)names.size();
  }
  {
    Deck f(dir + "/CONFIG", 54, "problem reading CONFIG file");
    f.next();
    Record r = f.next();
    r.take_int();
    d.imcon = r.take_int();
    for (int row = 0; row < 3; row++) {
      Record c = f.next();
      for (int j = 0; j < 3; j++) d.cell[3 * row + j] = c.take_double();
    }
  }
  double cp[10];
  cell_props(d.cell, cp);
  bool lcut = false, lrvdw = false;
  {
    Deck f(dir + "/CONTROL", 53, "end of CONTROL file encountered");
    for (;;) {
      Record r = f.next();
      r.lower();
      r.strip();
      if (r.blank_or_comment()) continue;
      if (r.has("cut")) {
        d.rcut = r.take_double();
        lcut = true;
      } else if (r.has("max guest atoms")) {
        d.maxguest = r.take_int();
      } else if (r.has("max framework atoms")) {
      } else if (r.has("&guest")) {
        s.nguest_control++;
        for (;;) {
          Record g = f.next();
          g.lower();
          g.strip();
          if (g.blank_or_comment()) continue;
          if (g.has("probability")) {
            int q = g.take_int(), seen = 0;
            while (seen < q) {
              Record p = f.next();
              p.strip();
              if (!p.blank_or_comment()) seen++;
            }
          } else if (g.has("&end")) {
            break;
          }
        }
      } else if (r.has("finishment")) {
      } else if (r.has("delr")) {
        d.delr = r.take_double();
      } else if (r.has("finish")) {
        break;
      } else if (r.has("ewald")) {
        s.lewald = true;
        d.keyfce = 2;
        if (r.has("precision")) {
          double eps = r.take_double();
          if (lcut) {
            // DL_POLY precision rule (utility_pack.f:381-391)
            eps = std::min(std::fabs(eps), 0.5);
            double tol = std::sqrt(std::fabs(std::log(eps * d.rcut)));
            d.alpha = std::sqrt(std::fabs(std::log(eps * d.rcut * tol))) / d.rcut;
            double t2 = 2.0 * tol * d.alpha;
            double tol1 = std::sqrt(-std::log(eps * d.rcut * (t2 * t2)));
            double fac = (d.imcon == 4 || d.imcon == 5 || d.imcon == 7) ? std::pow(2.0, 1.0 / 3.0) : 1.0;
            for (int i = 0; i < 3; i++) d.kmax[i] = (int)std::round(0.25 + fac * cp[i] * d.alpha * tol1 / 3.141592653589793);
          }
        } else {
          d.alpha = r.take_double();
          for (int i = 0; i < 3; i++) d.kmax[i] = r.take_int();
        }
      } else if (r.has("rvdw")) {
        d.rvdw = r.take_double();
        lrvdw = true;
      } else if (r.has("grid")) {
        // probability grid parameters (utility_pack.f:403-411)
        if (r.has("spa")) {
          d.griddim = r.take_double();
        } else if (r.has("fac")) {
          for (int i = 0; i < 3; i++) d.gridfactor[i] = r.take_int();
        }
      }
    }
  }
  if (d.rcut > half_width(d, cp)) raise(95, "potential cutoff exceeds half-cell width");
  d.volm = volume_of(d.imcon, cp);
  if (!lrvdw && d.rcut > 0.0) d.rvdw = d.rcut;
  if (!s.lewald) raise(2311, "GCMC sim needs ewald specified in CONTROL file");
}

// One FIELD molecule: a guest species (index into deck.guests) or a framework block.
struct MolBlock {
  bool guest;
  int index;  // guest index, or offset of the block's first atom in the framework arrays
  int nummols, numatoms;
  std::vector<std::string> names;
};

// ---------------------------------------------------------------- FIELD (readinputs.f:11-307)
void read_field(const std::string& dir, InputDeck& d, const Scan& s, std::vector<MolBlock>& blocks) {
  Deck f(dir + "/FIELD", 52, "end of FIELD file encountered");
  d.maxvdw = std::max(d.ntpvdw, (s.mxatyp * (s.mxatyp + 1)) / 2);
  d.mxgrid = std::max(1000, (int)(d.rvdw / 0.01 + 0.5) + 4);  // utility_pack.f:725
  d.ltpvdw.assign(d.maxvdw + 2, -1);
  d.lstvdw.assign(d.maxvdw + 2, 0);
  d.prmvdw.assign(d.maxvdw + 2, {0, 0, 0, 0, 0});
  f.next();
  for (;;) {
    Record r = f.next();
    r.lower();
    r.strip();
    if (r.has("units")) {
      bool blank = true;
      for (int i = 5; i < kRecLen; i++)
        if (r.c[i] != ' ') blank = false;
      if (blank) {
      } else if (r.has("ev")) d.engunit = 9648.530821;
      else if (r.has("kcal")) d.engunit = 418.4;
      else if (r.has("kj")) d.engunit = 1.0e2;
      else if (r.has("k")) d.engunit = 1.3806503e-23;
    } else if (r.has("vdw")) {
      // define_van_der_waals (vdw_terms.f:1-187)
      for (int itp = 1; itp <= d.ntpvdw; itp++) {
        Record v = f.next();
        std::string a1 = v.take_word(8), a2 = v.take_word(8);
        v.lower(kRecLen - 16);
        std::string kw = v.take_word(4).substr(0, 4);
        static const char* keys[] = {"tab ", "12-6", "lj  ", "nm  ", "buck", "bhm ", "hbnd", "snm ", "hcnm", "mors", "wca "};
        static const int keypots[] = {0, 1, 2, 3, 4, 5, 6, 7, 7, 8, 9};
        int keypot = -1;
        for (int k = 0; k < 11; k++)
          if (kw == keys[k]) keypot = keypots[k];
        std::array<double, 5> p;
        for (int i = 0; i < 5; i++) p[i] = v.take_double();
        int k1 = 0, k2 = 0;
        for (int j = 0; j < (int)d.types.size(); j++) {
          if (a1 == d.types[j]) k1 = j + 1;
          if (a2 == d.types[j]) k2 = j + 1;
        }
        if (k1 == 0 || k2 == 0) raise(4, "vdw pair names an unknown atom type");
        int hi = std::max(k1, k2), lo = std::min(k1, k2);
        int key = hi * (hi - 1) / 2 + lo;  // loc8, utility_pack.f:2386
        p[0] *= d.engunit;
        if (keypot == 1 || keypot == 6) p[1] *= d.engunit;
        if (keypot == 4) p[2] *= d.engunit;
        if (keypot == 5) {
          p[3] *= d.engunit;
          p[4] *= d.engunit;
        }
        d.lstvdw[key] = itp;
        d.ltpvdw[itp] = keypot;
        d.prmvdw[itp] = p;
      }
      int ntab = (int)(d.types.size() * (d.types.size() + 1) / 2);
      if (d.ntpvdw < ntab)
        for (int i = 1; i <= ntab; i++)
          if (d.lstvdw[i] == 0) d.lstvdw[i] = d.ntpvdw + 1;
    } else if (r.has("molecu")) {
      int nmt = r.take_int();
      for (int n = 0; n < nmt; n++) {
        Record h = f.next();
        h.lower();
        bool guest = h.has("&guest");
        if (guest) h.take_word(6);  // the species name follows the keyword (readinputs.f:131-141)
        h.strip();
        int nummols = 0, numatoms = 0;
        std::vector<std::string> names;
        std::vector<double> mass, chg, gx, gy, gz;
        std::vector<int> frz, typ;
        for (;;) {
          Record m = f.next();
          m.lower();
          m.strip();
          if (m.has("nummol")) {
            nummols = m.take_int();
          } else if (m.has("atoms")) {
            numatoms = m.take_int();
            names.assign(numatoms, "");
            mass.assign(numatoms, 0);
            chg.assign(numatoms, 0);
            frz.assign(numatoms, 0);
            typ.assign(numatoms, 0);
            gx.assign(numatoms, 0);
            gy.assign(numatoms, 0);
            gz.assign(numatoms, 0);
            int ksite = 0;
            for (int isite = 0; isite < numatoms; isite++) {
              if (ksite >= numatoms) continue;
              Record a = f.next();  // atom records keep their case (readinputs.f:176-180)
              std::string name = a.take_word(8);
              double w = a.take_double(), q = a.take_double();
              int nrept = 1, ifrz = 0;
              if (guest) {
                gx[isite] = a.take_double();
                gy[isite] = a.take_double();
                gz[isite] = a.take_double();
              } else {
                nrept = a.take_int();
                ifrz = a.take_int();
              }
              if (nrept == 0) nrept = 1;
              if (ksite + nrept > numatoms) raise(4, "atom repeat count overruns the ATOMS block");
              int tix = 0;
              for (int j = 0; j < (int)d.types.size(); j++)
                if (d.types[j] == name) tix = j + 1;
              if (tix == 0) {
                d.types.push_back(name);
                tix = (int)d.types.size();
              }
              for (int k = 0; k < nrept; k++, ksite++) {
                names[ksite] = name;
                mass[ksite] = w;
                chg[ksite] = q;
                frz[ksite] = ifrz;
                typ[ksite] = tix;
              }
            }
          } else if (m.has("finish")) {
            break;
          }
        }
        MolBlock b{guest, 0, nummols, numatoms, names};
        if (guest) {
          double M = 0, cx = 0, cy = 0, cz = 0;
          for (int i = 0; i < numatoms; i++) {
            cx = cx + gx[i] * mass[i];
            cy = cy + gy[i] * mass[i];
            cz = cz + gz[i] * mass[i];
            M = M + mass[i];
          }
          cx = cx / M;
          cy = cy / M;
          cz = cz / M;
          for (int i = 0; i < numatoms; i++) {
            gx[i] -= cx;
            gy[i] -= cy;
            gz[i] -= cz;
          }
          if (numatoms > 50) raise(75, "guest has more sites than the 50-site limit");
          GuestSpecies g;
          g.name = std::string(h.c, 40);
          g.nsite = numatoms;
          g.site_name = names;
          g.mass = mass;
          g.charge = chg;
          g.tx = gx;
          g.ty = gy;
          g.tz = gz;
          g.type = typ;
          g.nmols = nummols;
          b.index = (int)d.guests.size();
          d.guests.push_back(g);
        } else {
          b.index = (int)d.fq.size();
          for (int im = 0; im < nummols; im++)
            for (int k = 0; k < numatoms; k++) {
              d.fq.push_back(chg[k]);
              d.ftype.push_back(typ[k]);
              d.ffrz.push_back(frz[k]);
              d.fname.push_back(names[k]);
              d.fmass.push_back(mass[k]);
            }
        }
        blocks.push_back(b);
      }
    } else if (r.has("close")) {
      break;
    } else {
      raise(4, "unknown directive found in FIELD file");
    }
  }
}

// Fortran '(3f20.0)' read: three 20-character numeric fields
double f20(std::string_view s, int k) {
  char t[24];
  int n = 0;
  for (int i = 20 * k; i < 20 * k + 20 && i < (int)s.size(); i++) {
    char ch = s[i];
    if (ch == ' ' || ch == '\r' || ch == '\t') continue;
    t[n++] = ch == 'd' || ch == 'D' ? 'e' : ch;
  }
  t[n] = 0;
  if (!n) return 0.0;
  // std::from_chars rounds correctly, as strtod does, and is several times faster; strtod keeps
  // what from_chars does not read the same way (a leading '+', hexadecimal, out of range)
  if (t[0] != '+' && !std::memchr(t, 'x', n) && !std::memchr(t, 'X', n)) {
    double v = 0.0;
    const std::from_chars_result r = std::from_chars(t, t + n, v);
    if (r.ec == std::errc()) return v;
  }
  return std::strtod(t, nullptr);
}

// ---------------------------------------------------------------- CONFIG (readinputs.f:309-513)
void read_config(const std::string& dir, InputDeck& d, const std::vector<MolBlock>& blocks) {
  Deck f(dir + "/CONFIG", 54, "problem reading CONFIG file");
  f.next();
  Record h = f.next();
  int levcfg = h.take_int();
  if (d.imcon == 0) {
    for (double& c : d.cell) c = 0.0;
  } else {
    for (int row = 0; row < 3; row++) {
      Record c = f.next();
      for (int j = 0; j < 3; j++) d.cell[3 * row + j] = c.take_double();
    }
  }
  d.fx.assign(d.fq.size(), 0.0);
  d.fy.assign(d.fq.size(), 0.0);
  d.fz.assign(d.fq.size(), 0.0);
  for (const MolBlock& b : blocks) {
    std::vector<double>* gxyz = b.guest ? &d.guests[b.index].xyz : nullptr;
    if (gxyz) gxyz->assign(3 * b.nummols * b.numatoms, 0.0);
    int at = 0;
    for (int l = 0; l < b.nummols; l++)
      for (int m = 0; m < b.numatoms; m++, at++) {
        const std::string_view name_line = f.raw();
        const std::string_view coord_line = f.raw();
        for (int e = 0; e < levcfg; e++) f.raw();
        // the first 8 characters, leading blanks dropped, blank-padded to 8
        std::string_view an = name_line.substr(0, std::min<size_t>(8, name_line.size()));
        const size_t k = an.find_first_not_of(' ');
        an = k == std::string_view::npos ? std::string_view() : an.substr(k);
        const std::string& want = b.names[m];
        if (want.size() != 8 || want.compare(0, an.size(), an) != 0 ||
            want.find_first_not_of(' ', an.size()) != std::string::npos)
          raise(25, "wrong atom type found in CONFIG file");
        double x = f20(coord_line, 0), y = f20(coord_line, 1), z = f20(coord_line, 2);
        if (gxyz) {
          (*gxyz)[3 * at] = x;
          (*gxyz)[3 * at + 1] = y;
          (*gxyz)[3 * at + 2] = z;
        } else {
          d.fx[b.index + at] = x;
          d.fy[b.index + at] = y;
          d.fz[b.index + at] = z;
        }
      }
  }
  const double* c = d.cell;
  auto bad = [] { raise(410, "cell not consistent with image convention"); };
  if (d.imcon == 1 || d.imcon == 4 || d.imcon == 5) {
    double axx = (std::fabs(c[0]) + std::fabs(c[4])) / 2.0, test = 1e-8 * axx;
    if (std::fabs(c[0] - axx) > test || std::fabs(c[4] - axx) > test) bad();
    double want = d.imcon == 5 ? axx * std::sqrt(2.0) : axx;
    if (std::fabs(c[8] - want) > test) bad();
  }
  if (d.imcon == 7 && std::fabs(c[0] - std::sqrt(3.0) * c[4]) >= 1e-6) bad();
  if (d.imcon == 6 && (std::fabs(c[2]) > 1e-10 || std::fabs(c[5]) > 1e-10 || std::fabs(c[6]) > 1e-10 ||
                       std::fabs(c[7]) > 1e-10))
    bad();
  if (d.imcon == 1 || d.imcon == 2 || d.imcon == 4 || d.imcon == 5 || d.imcon == 7)
    for (int i : {1, 2, 3, 5, 6, 7})
      if (std::fabs(c[i]) > 1e-10) bad();
  double cp[10];
  cell_props(d.cell, cp);
  d.volm = volume_of(d.imcon, cp);
  if (d.imcon > 0 && d.rcut > half_width(d, cp)) raise(95, "potential cutoff exceeds half-cell width");
}

// ---------------------------------------------------------------- CONTROL (readinputs.f:515-914)
void read_control(const std::string& dir, InputDeck& d) {
  Deck f(dir + "/CONTROL", 53, "end of CONTROL file encountered");
  const int ng = (int)d.guests.size();
  d.press.assign(ng, 0.0);
  d.adspres.assign(ng, 0.0);
  d.adsguen.assign(ng, 0.0);
  d.movefreq.assign(ng, {0, 0, 0, 0, 0, 0, 0, 0, 0});
  d.disp_ratio.assign(ng, 0.5);
  d.tran_ratio.assign(ng, 0.5);
  std::vector<char> own_moves(ng, 0), own_disp(ng, 0), own_tran(ng, 0);
  bool ltemp = false, lsteps = false, leq = false, lwind = false, lnumg = false;
  int nblocks = 0;
  // move keyword -> slot, tested in the reference's order (readinputs.f:649-667, 785-834)
  static const char* mv_keys[] = {"ins", "del", "dis", "jum", "fle", "swa", "tra", "rot", "mul"};
  f.next();
  for (;;) {
    Record r = f.next();
    r.lower();
    r.strip();
    if (r.blank_or_comment()) continue;
    if (r.has("restart")) {
      d.lrestart = true;
    } else if (r.has("temp")) {
      d.temp = r.take_double();
      ltemp = true;
    } else if (r.has("sampling")) {
      d.laccsample = true;
    } else if (r.has("&guest")) {
      nblocks++;
      Record outer = r;  // the per-guest 'delr' test reads this record (readinputs.f:686)
      int id = r.take_int();
      if (id < 1 || id > ng) raise(2312, "&guest index does not match the FIELD guests");
      int g = id - 1;
      for (;;) {
        Record q = f.next();
        q.lower();
        q.strip();
        if (q.blank_or_comment()) continue;
        if (q.has("fract")) {
          q.take_double();
        } else if (q.has("press")) {
          d.press[g] = q.take_double() * 1.0e5;
        } else if (q.has("probability")) {
          // probability plots of this guest: per plot, a site count then the sites (0: the
          // molecule's centre of mass) (readinputs.f:638-660)
          int n = q.take_int(), seen = 0;
          while (seen < n) {
            Record p = f.next();
            p.strip();
            if (p.blank_or_comment()) continue;
            seen++;
            ProbPlot plot;
            plot.guest = g;
            int ns = p.take_int();
            for (int j = 0; j < ns; j++) plot.sites.push_back(p.take_int());
            d.plots.push_back(plot);
          }
        } else if (q.has("move")) {
          own_moves[g] = 1;
          for (int k = 0; k < 9; k++)
            if (q.has(mv_keys[k])) {
              d.movefreq[g][k] = q.take_double();
              break;
            }
        } else if (outer.has("delr")) {
          q.take_double();  // per-guest delr never reaches the module array
        } else if (q.has("accep")) {
          if (q.has("dis")) {
            own_disp[g] = 1;
            d.disp_ratio[g] = q.take_double();
          } else if (q.has("tra")) {
            own_tran[g] = 1;
            d.tran_ratio[g] = q.take_double();
          }
        } else if (q.has("&end")) {
          break;
        }
      }
    } else if (r.has("steps")) {
      d.mcsteps = r.take_int();
      lsteps = true;
    } else if (r.has("pressure") || r.has("total press")) {
    } else if (r.has("numg")) {
      d.nnumg = r.take_int();
      if (d.nnumg <= 0) d.nnumg = 1000;
      lnumg = true;
    } else if (r.has("fuga")) {
    } else if (r.has("hist")) {
      d.nhis = r.take_int();
    } else if (r.has("equilibr")) {
      d.eqsteps = r.take_int();
      leq = d.eqsteps != 0;
    } else if (r.has("uvt")) {
    } else if (r.has("single point")) {
      d.lspe = true;
    } else if (r.has("jobcontrol")) {
    } else if (r.has("cutoff")) {
      d.rcut = r.take_double();
    } else if (r.has("delr")) {
    } else if (r.has("ewald")) {
    } else if (r.has("averaging window")) {
      d.nwind = r.take_int();
      lwind = true;
    } else if (r.has("max guest atoms")) {
      d.maxguest = r.take_int();
    } else if (r.has("max framework atoms")) {
    } else if (r.has("desorb")) {
      d.desorb = r.take_int();
    } else if (r.has("adsorb press")) {
      for (int i = 0; i < ng; i++) d.adspres[i] = r.take_double();
    } else if (r.has("adsorb guests")) {
      for (int i = 0; i < ng; i++) d.adsguen[i] = r.take_double();
    } else if (r.has("packing fraction")) {
      d.packf = r.take_double();
    } else if (r.has("finishment")) {
      d.despre = r.take_double();
    } else if (r.has("move")) {
      for (int k = 0; k < 9; k++)
        if (r.has(mv_keys[k])) {
          double v = r.take_double();
          for (int g = 0; g < ng; g++)
            if (!own_moves[g]) d.movefreq[g][k] = v;
          break;
        }
    } else if (r.has("accep")) {
      if (r.has("dis")) {
        double v = r.take_double();
        for (int g = 0; g < ng; g++)
          if (!own_disp[g]) d.disp_ratio[g] = v;
      } else if (r.has("tra")) {
        double v = r.take_double();
        for (int g = 0; g < ng; g++)
          if (!own_tran[g]) d.tran_ratio[g] = v;
      } else if (r.has("rot")) {
        d.rota_ratio = r.take_double();
      }
    } else if (r.has("grid")) {
    } else if (r.has("finish")) {
      break;
    } else {
      raise(3, "unknown directive found in CONTROL file");
    }
  }
  if (!leq) d.eqsteps = 0;
  if (!lnumg) d.nnumg = d.eqsteps > 1000 ? d.eqsteps / 1000 : 1;
  if (d.despre > 0) {
    // the reference allocates its work array only for desorb 1 and indexes the per-guest arrays
    // by FIELD molecule index (gcmc.f:275-281, 655-679)
    if (d.desorb != 1) raise(-2, "finishment needs desorb 1");
  }
  if (!lsteps) {
    d.mcsteps = 1;
    d.lspe = true;
  }
  if (!lwind) d.nwind = 100000;
  if (nblocks != ng) raise(2312, "number of &guest blocks differs from the FIELD guests");
  if (!ltemp) raise(380, "simulation temperature not specified");
}

}  // namespace

int finish_deck_from_arrays(InputDeck& d, std::string& err) {
  try {
    const int nt = (int)d.types.size();
    if (d.imcon < 1 || d.imcon > 7) raise(-4, "the device path needs periodic boundaries (imcon 1-7)");
    if (!(d.rcut > 0.0)) raise(-1, "cut-off must be positive");
    if (!(d.alpha > 0.0) || d.kmax[0] < 1 || d.kmax[1] < 1 || d.kmax[2] < 1)
      raise(2311, "GCMC sim needs ewald (alpha and kmax) specified");
    if (nt < 1) raise(4, "no atom types");
    const double* c = d.cell;
    auto bad = [] { raise(410, "cell not consistent with image convention"); };
    if (d.imcon == 1 || d.imcon == 4 || d.imcon == 5) {
      double axx = (std::fabs(c[0]) + std::fabs(c[4])) / 2.0, test = 1e-8 * axx;
      if (std::fabs(c[0] - axx) > test || std::fabs(c[4] - axx) > test) bad();
      double want = d.imcon == 5 ? axx * std::sqrt(2.0) : axx;
      if (std::fabs(c[8] - want) > test) bad();
    }
    if (d.imcon == 7 && std::fabs(c[0] - std::sqrt(3.0) * c[4]) >= 1e-6) bad();
    if (d.imcon == 6 && (std::fabs(c[2]) > 1e-10 || std::fabs(c[5]) > 1e-10 || std::fabs(c[6]) > 1e-10 ||
                         std::fabs(c[7]) > 1e-10))
      bad();
    if (d.imcon == 1 || d.imcon == 2 || d.imcon == 4 || d.imcon == 5 || d.imcon == 7)
      for (int i : {1, 2, 3, 5, 6, 7})
        if (std::fabs(c[i]) > 1e-10) bad();
    double cp[10];
    cell_props(d.cell, cp);
    d.volm = volume_of(d.imcon, cp);
    if (d.rcut > half_width(d, cp)) raise(95, "potential cutoff exceeds half-cell width");
    if (!(d.rvdw > 0.0)) d.rvdw = d.rcut;
    d.keyfce = 2;
    d.maxvdw = std::max(d.ntpvdw, (nt * (nt + 1)) / 2);
    d.mxgrid = std::max(1000, (int)(d.rvdw / 0.01 + 0.5) + 4);  // utility_pack.f:725
    // pair tables: every pair without a line of its own gets the zero table (vdw_terms.f:160-182)
    if ((int)d.ltpvdw.size() != d.ntpvdw + 1 || (int)d.prmvdw.size() != d.ntpvdw + 1 ||
        (int)d.lstvdw.size() != (nt * (nt + 1)) / 2 + 1)
      raise(-1, "vdW tables sized inconsistently with the pair count");
    d.ltpvdw.resize(d.maxvdw + 2, -1);
    d.prmvdw.resize(d.maxvdw + 2, {0, 0, 0, 0, 0});
    d.lstvdw.resize(d.maxvdw + 2, 0);
    const int ntab = nt * (nt + 1) / 2;
    if (d.ntpvdw < ntab)
      for (int i = 1; i <= ntab; i++)
        if (d.lstvdw[i] == 0) d.lstvdw[i] = d.ntpvdw + 1;
    for (int t : d.ftype)
      if (t < 1 || t > nt) raise(4, "framework atom of an unknown type");
    for (const GuestSpecies& g : d.guests) {
      if (g.nsite < 1 || g.nsite > 50) raise(75, "guest site count outside 1-50");
      for (int t : g.type)
        if (t < 1 || t > nt) raise(4, "guest site of an unknown type");
    }
    if (d.temp <= 0.0) raise(380, "simulation temperature not specified");
    d.nnumg = d.eqsteps > 1000 ? d.eqsteps / 1000 : 1;
    return 0;
  } catch (const InputError& e) {
    err = e.msg;
    return e.code;
  }
}

int read_input_deck(const std::string& dir, InputDeck& d, std::string& err) {
  try {
    d = InputDeck();
    Scan s;
    prescan(dir, d, s);
    std::vector<MolBlock> blocks;
    read_field(dir, d, s, blocks);
    read_config(dir, d, blocks);
    read_control(dir, d);
    for (const MolBlock& b : blocks)
      d.mols.push_back({b.guest ? b.index : -1, b.guest ? 0 : b.index, b.nummols, b.numatoms});
    // pressure equilibration indexes the per-guest arrays by FIELD molecule index (gcmc.f:655-679)
    if (d.despre > 0)
      for (size_t i = 0; i < d.guests.size(); i++)
        if (i >= d.mols.size() || d.mols[i].guest != (int)i)
          raise(-2, "pressure equilibration needs the guests first in FIELD");
    if (!d.plots.empty()) {  // gcmc.f:246-256
      double cp[10];
      cell_props(d.cell, cp);
      for (int i = 0; i < 3; i++)
        d.ngrid[i] = d.gridfactor[i] * (int)std::ceil(cp[i] / (d.griddim * d.gridfactor[i]));
      for (const ProbPlot& pl : d.plots)
        for (int site : pl.sites)
          if (site < 0 || site > d.guests[pl.guest].nsite) raise(-4, "probability plot names a site the guest lacks");
    }
    {
      std::ifstream f(dir + "/CONFIG");
      std::getline(f, d.title);
      if (!d.title.empty() && d.title.back() == '\r') d.title.pop_back();
    }
    return 0;
  } catch (const InputError& e) {
    err = e.msg;
    return e.code;
  }
}

}  // namespace fmc
