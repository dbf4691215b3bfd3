// TEST INFRASTRUCTURE ONLY -- never linked into, called by, or shipped with the product.
//
// FP64 CPU restatement ("oracle") of FastMC 1.4.0's GCMC trial-move energy path, used by
// tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg as the checker and as the
// timed CPU baseline ("port" kind).  The reference is Fortran and cannot be compiled in this
// image (no Fortran compiler), so parity is pinned by the reference's own shipped outputs:
//   * examples/restart/1_*/OUTPUT:113   "Energy reported by DL_POLY: -11190.606165"
//     (empty CALF-20 framework, reciprocal + self energy), and
//   * examples/restart/1_*/branch01/REVIVE  energy(1) = -731.5072668178669 kcal/mol
//     (a loose pin: that number is a running sum over 2.26e8 accepted moves).
// Every routine below cites the reference file:line it restates, keeps the reference's
// loop order, and is compiled with -O2 -ffp-contract=off (no FMA contraction, like a
// plain x86-64 gfortran build).  Indices are 0-based here; the citations are 1-based.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

namespace orc {

// utility_pack.f:77-113 constants
static const double PI = 3.141592653589793;
static const double SQRPI = 1.7724538509055159;
static const double R4PIE0 = 138935.4835;
static const double KBOLTZ = 1.9872041e-3;
static const double BOLTZ = 1.3806503e-23;
static const double RGAS = 8.314472 / 4184.0;
// calc_Qst, calc_Cv (utility_pack.f:2280-2316)
static double calc_qst(double E2, double E, double N, double N2, double EN, double temp) {
  (void)E2;
  return -1.0 * (EN - E * N) / (N2 - N * N) + RGAS * temp;
}
static double calc_cv(double E2, double E, double N, double N2, double EN, double temp) {
  const double d = EN - E * N;
  return (3.0 / 2.0 * RGAS) + (E2 - (E * E) - d * d / (N2 - N * N)) / (N * KBOLTZ * temp * temp);
}
static const double MINANGLE = PI / 18.0;
static const double DELRMIN = 0.1;
static const int LENREC = 150;

struct FmcError {
  int code;
  std::string msg;
};
[[noreturn]] static void fail(int code, const std::string& msg) { throw FmcError{code, msg}; }

// ---------------------------------------------------------------- parse_module.f
// A record is a 150-character, blank-padded line (parse_module.f:16-18, getrec 22-95).
struct Rec {
  char c[LENREC];
};

class LineFile {
 public:
  explicit LineFile(const std::string& path) {
    std::ifstream f(path);
    if (!f) fail(-1, "cannot open " + path);
    std::string s;
    while (std::getline(f, s)) {
      if (!s.empty() && s.back() == '\r') s.pop_back();
      lines_.push_back(s);
    }
  }
  bool getrec(Rec& r) {
    if (pos_ >= lines_.size()) return false;
    const std::string& s = lines_[pos_++];
    for (int i = 0; i < LENREC; i++) r.c[i] = i < (int)s.size() ? s[i] : ' ';
    for (int i = 0; i < LENREC; i++)
      if (r.c[i] == '\t') r.c[i] = ' ';
    return true;
  }
  bool rawline(std::string& s) {
    if (pos_ >= lines_.size()) return false;
    s = lines_[pos_++];
    return true;
  }

 private:
  std::vector<std::string> lines_;
  size_t pos_ = 0;
};

// lowcase parse_module.f:331-420
static void lowcase(char* s, int n) {
  for (int i = 0; i < n && i < 255; i++)
    if (s[i] >= 'A' && s[i] <= 'Z') s[i] = s[i] - 'A' + 'a';
}
// strip parse_module.f:290-329: drop leading blanks
static void strip(char* s, int n) {
  for (int i = 0; i < n; i++) {
    if (s[0] == ' ') {
      for (int j = 0; j < n - 1; j++) s[j] = s[j + 1];
      s[n - 1] = ' ';
    }
  }
}
// findstring parse_module.f:449-492
static bool findstring(const char* seek, const char* s) {
  int n = (int)strlen(seek);
  for (int here = 0; here <= LENREC - n; here++)
    if (strncmp(seek, s + here, n) == 0) return true;
  return false;
}
static void shift_word(char* w, int len, int lst) {
  // parse_module.f:158-163: word(j-lst+1)=word(j), j=lst..len; blank the tail
  for (int j = lst; j <= len; j++) w[j - lst] = w[j - 1];
  for (int j = len - lst + 2; j <= len; j++) w[j - 1] = ' ';
}
// intstr parse_module.f:96-170
static int intstr(char* w, int len, int* lst_out) {
  int isn = 1, lst = 0, v = 0;
  char ksn = '+';
  bool flag = false, fin = false, count = false;
  while (lst < len && !fin) {
    lst++;
    flag = false;
    char ch = w[lst - 1];
    if (ch >= '0' && ch <= '9') {
      v = 10 * v + (ch - '0');
      count = true;
      flag = true;
    }
    if (count && !flag) fin = true;
    if (flag && ksn == '-') isn = -1;
    ksn = ch;
  }
  v = isn * v;
  shift_word(w, len, lst);
  if (lst_out) *lst_out = lst;
  return v;
}
// libgcc __powidf2: what gfortran emits for real(8)**integer
static double powi(double x, int m) {
  unsigned n = m < 0 ? -(unsigned)m : (unsigned)m;
  double y = (n % 2) ? x : 1.0;
  while (n >>= 1) {
    x = x * x;
    if (n % 2) y = y * x;
  }
  return m < 0 ? 1.0 / y : y;
}
// dblstr parse_module.f:171-289 (digit-by-digit accumulation, not strtod)
static double dblstr(char* w, int len) {
  int lst = 0, iexp = 0, idum = 0;
  double sn = 1.0, ten = 10.0, one = 1.0, v = 0.0;
  char ksn = '+';
  bool start = false, ldot = false, fin = false;
  std::vector<char> work(len + 1, ' ');
  while (lst < len && !fin) {
    lst++;
    bool flag = false;
    char ch = w[lst - 1];
    if (ch >= '0' && ch <= '9') {
      v = ten * v + one * (double)(ch - '0');
      flag = true;
      start = true;
    }
    if (ch == '.') {
      flag = true;
      ten = 1.0;
      ldot = true;
      start = true;
    }
    if (flag && ksn == '-') sn = -1.0;
    if (ldot) one = one / 10.0;
    ksn = ch;
    if (ksn == 'D') ksn = 'd';
    if (ksn == 'E') ksn = 'e';
    if (start) {
      if (ksn == 'd' || ksn == 'e') {
        for (int i = 1; i <= len - lst; i++) work[i - 1] = w[i + lst - 1];
        iexp = intstr(work.data(), len - lst, &idum);
        fin = true;
      }
      if (!flag) fin = true;
    }
  }
  v = sn * v * powi(10.0, iexp);
  lst = lst + idum;
  shift_word(w, len, lst);
  return v;
}
// getword parse_module.f:547-603; returns the word blank-padded to 8 characters
static std::string getword(char* s, int len1, int len2) {
  char seq[64];
  for (int i = 0; i < 64; i++) seq[i] = ' ';
  int i = 0, k = 0;
  bool fin = false;
  while (!fin && i < len2) {
    i++;
    if (s[0] == ' ') {
      if (k > 0) fin = true;
    } else {
      k++;
      seq[k - 1] = s[0];
      if (k == len1) fin = true;
    }
    for (int j = 0; j < len2 - 1; j++) s[j] = s[j + 1];
    s[len2 - 1] = ' ';
  }
  return std::string(seq, 8);
}

// ---------------------------------------------------------------- geometry (utility_pack.f)
// invert utility_pack.f:1417-1467
static void invert(const double* a, double* b, double* d) {
  b[0] = a[4] * a[8] - a[5] * a[7];
  b[1] = a[2] * a[7] - a[1] * a[8];
  b[2] = a[1] * a[5] - a[2] * a[4];
  b[3] = a[5] * a[6] - a[3] * a[8];
  b[4] = a[0] * a[8] - a[2] * a[6];
  b[5] = a[2] * a[3] - a[0] * a[5];
  b[6] = a[3] * a[7] - a[4] * a[6];
  b[7] = a[1] * a[6] - a[0] * a[7];
  b[8] = a[0] * a[4] - a[1] * a[3];
  *d = a[0] * b[0] + a[3] * b[1] + a[6] * b[2];
  double r = 0.0;
  if (std::fabs(*d) > 0.0) r = 1.0 / *d;
  for (int i = 0; i < 9; i++) b[i] = r * b[i];
}
// dcell utility_pack.f:1351-1415
static void dcell(const double* a, double* b) {
  b[0] = std::sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
  b[1] = std::sqrt(a[3] * a[3] + a[4] * a[4] + a[5] * a[5]);
  b[2] = std::sqrt(a[6] * a[6] + a[7] * a[7] + a[8] * a[8]);
  b[3] = (a[0] * a[3] + a[1] * a[4] + a[2] * a[5]) / (b[0] * b[1]);
  b[4] = (a[0] * a[6] + a[1] * a[7] + a[2] * a[8]) / (b[0] * b[2]);
  b[5] = (a[3] * a[6] + a[4] * a[7] + a[5] * a[8]) / (b[1] * b[2]);
  double axb1 = a[1] * a[5] - a[2] * a[4];
  double axb2 = a[2] * a[3] - a[0] * a[5];
  double axb3 = a[0] * a[4] - a[1] * a[3];
  double bxc1 = a[4] * a[8] - a[5] * a[7];
  double bxc2 = a[5] * a[6] - a[3] * a[8];
  double bxc3 = a[3] * a[7] - a[4] * a[6];
  double cxa1 = a[7] * a[2] - a[1] * a[8];
  double cxa2 = a[0] * a[8] - a[2] * a[6];
  double cxa3 = a[1] * a[6] - a[0] * a[7];
  b[9] = std::fabs(a[0] * bxc1 + a[1] * bxc2 + a[2] * bxc3);
  b[6] = b[9] / std::sqrt(bxc1 * bxc1 + bxc2 * bxc2 + bxc3 * bxc3);
  b[7] = b[9] / std::sqrt(cxa1 * cxa1 + cxa2 * cxa2 + cxa3 * cxa3);
  b[8] = b[9] / std::sqrt(axb1 * axb1 + axb2 * axb2 + axb3 * axb3);
}
// Fortran nint: round half away from zero
static inline double fnint(double x) { return std::round(x); }
static inline double fsign(double a, double b) { return b >= 0.0 ? std::fabs(a) : -std::fabs(a); }

// images utility_pack.f:1138-1349 (all imcon branches)
static void images(int imcon, int n, const double* cell, double* x, double* y, double* z) {
  const double rt2 = 1.41421356623, rt3 = 1.7320508075;
  if (imcon == 1) {
    double aaa = 1.0 / cell[0];
    for (int i = 0; i < n; i++) {
      x[i] = x[i] - cell[0] * fnint(aaa * x[i]);
      y[i] = y[i] - cell[0] * fnint(aaa * y[i]);
      z[i] = z[i] - cell[0] * fnint(aaa * z[i]);
    }
  } else if (imcon == 2) {
    double aaa = 1.0 / cell[0], bbb = 1.0 / cell[4], ccc = 1.0 / cell[8];
    for (int i = 0; i < n; i++) {
      x[i] = x[i] - cell[0] * fnint(aaa * x[i]);
      y[i] = y[i] - cell[4] * fnint(bbb * y[i]);
      z[i] = z[i] - cell[8] * fnint(ccc * z[i]);
    }
  } else if (imcon == 3) {
    double rc[9], det;
    invert(cell, rc, &det);
    for (int i = 0; i < n; i++) {
      double ssx = (rc[0] * x[i] + rc[3] * y[i] + rc[6] * z[i]);
      double ssy = (rc[1] * x[i] + rc[4] * y[i] + rc[7] * z[i]);
      double ssz = (rc[2] * x[i] + rc[5] * y[i] + rc[8] * z[i]);
      double xss = ssx - fnint(ssx), yss = ssy - fnint(ssy), zss = ssz - fnint(ssz);
      x[i] = (cell[0] * xss + cell[3] * yss + cell[6] * zss);
      y[i] = (cell[1] * xss + cell[4] * yss + cell[7] * zss);
      z[i] = (cell[2] * xss + cell[5] * yss + cell[8] * zss);
    }
  } else if (imcon == 4) {
    double aaa = 1.0 / cell[0];
    for (int i = 0; i < n; i++) {
      x[i] = x[i] - cell[0] * fnint(aaa * x[i]);
      y[i] = y[i] - cell[0] * fnint(aaa * y[i]);
      z[i] = z[i] - cell[0] * fnint(aaa * z[i]);
      if ((std::fabs(x[i]) + std::fabs(y[i]) + std::fabs(z[i])) >= (0.75 * cell[0])) {
        x[i] = x[i] - 0.5 * fsign(cell[0], x[i]);
        y[i] = y[i] - 0.5 * fsign(cell[0], y[i]);
        z[i] = z[i] - 0.5 * fsign(cell[0], z[i]);
      }
    }
  } else if (imcon == 5) {
    double aaa = 1.0 / cell[0], bbb = 1.0 / cell[8];
    for (int i = 0; i < n; i++) {
      x[i] = x[i] - cell[0] * fnint(aaa * x[i]);
      y[i] = y[i] - cell[0] * fnint(aaa * y[i]);
      z[i] = z[i] - cell[8] * fnint(bbb * z[i]);
      if ((std::fabs(x[i]) + std::fabs(y[i]) + std::fabs(rt2 * z[i])) >= cell[0]) {
        x[i] = x[i] - 0.5 * fsign(cell[0], x[i]);
        y[i] = y[i] - 0.5 * fsign(cell[0], y[i]);
        z[i] = z[i] - 0.5 * fsign(cell[8], z[i]);
      }
    }
  } else if (imcon == 6) {
    double det = cell[0] * cell[4] - cell[1] * cell[3];
    det = 1.0 / det;
    double r1 = det * cell[4], r2 = -det * cell[1], r4 = -det * cell[3], r5 = det * cell[0];
    for (int i = 0; i < n; i++) {
      double ssx = r1 * x[i] + r4 * y[i];
      double ssy = r2 * x[i] + r5 * y[i];
      double xss = ssx - fnint(ssx), yss = ssy - fnint(ssy);
      x[i] = cell[0] * xss + cell[3] * yss;
      y[i] = cell[1] * xss + cell[4] * yss;
    }
  } else if (imcon == 7) {
    double aaa = cell[0] / (rt3 * 2.0), bbb = cell[0] / rt3, ccc = rt3 / cell[0], ddd = 1.0 / cell[8];
    for (int i = 0; i < n; i++) {
      y[i] = y[i] - bbb * fnint(ccc * y[i]);
      z[i] = z[i] - cell[8] * fnint(ddd * z[i]);
      if ((std::fabs(y[i]) + std::fabs(rt3 * x[i])) >= bbb) {
        x[i] = x[i] - rt3 * fsign(aaa, x[i]);
        y[i] = y[i] - fsign(aaa, y[i]);
      }
    }
  }
}

// ---------------------------------------------------------------- duni (gcmc.f:2712-2805)
// Marsaglia-Zaman-Tsang universal generator in REAL(4).  The seed (i,j,k,l) is injected
// instead of being derived from the wall clock (gcmc.f:2753-2758).  The reference's first
// call only initialises; the program then discards two calls (gcmc.f:335-336), so after
// construction one real draw is consumed here.
struct Duni {
  float u[97];
  float c, cd, cm;
  int ir, jr;
  void seed(int i, int j, int k, int l) {
    ir = 97;
    jr = 33;
    for (int ii = 0; ii < 97; ii++) {
      float s = 0.0f, t = 0.5f;
      for (int jj = 0; jj < 24; jj++) {
        int m = ((i * j) % 179) * k % 179;
        i = j;
        j = k;
        k = m;
        l = (53 * l + 1) % 169;
        if ((l * m) % 64 >= 32) s = s + t;
        t = 0.5f * t;
      }
      u[ii] = s;
    }
    c = 362436.0f / 16777216.0f;
    cd = 7654321.0f / 16777216.0f;
    cm = 16777213.0f / 16777216.0f;
  }
  double next() {
    float uni = u[ir - 1] - u[jr - 1];
    if (uni < 0.0f) uni = uni + 1.0f;
    u[ir - 1] = uni;
    ir = ir - 1;
    if (ir == 0) ir = 97;
    jr = jr - 1;
    if (jr == 0) jr = 97;
    c = c - cd;
    if (c < 0.0f) c = c + cm;
    uni = uni - c;
    if (uni < 0.0f) uni = uni + 1.0f;
    return (double)uni;
  }
};

// ---------------------------------------------------------------- system state
struct MolType {
  std::string name;
  bool guest = false;
  int nummols = 0, numatoms = 0;
  std::vector<std::string> atmname;
  std::vector<double> wght, chg;
  std::vector<int> frz, ltpsit;  // ltpsit 1-based unique type index
  std::vector<double> fx, fy, fz;  // framwkxxx(mol, 1..nummols*numatoms)
};

struct MoveRec {
  int32_t step, iguest, mtype, randchoice, accepted, nmols_after, pad0, pad1;
  double ewld1, ewld2, ewld3, vdw, delrc, estep, rande, energy_after;
};

struct ProbPlotO {
  int guest = 0;
  std::vector<int> sites;  // 0: centre of mass
};

struct Chain {
  // ---- probability plots (readinputs.f:638-660, gcmc.f:246-265, storeprob utility_pack.f:496-561)
  std::vector<ProbPlotO> plots;
  double griddim = 0.1;            // gcmc.f:136
  int gridfactor[3] = {1, 1, 1};   // gcmc.f:138
  int ngrid[3] = {0, 0, 0};
  std::vector<std::vector<double>> grid;  // [plot][a*nb*nc + b*nc + c]
  // ---- initscan (utility_pack.f:176-457)
  int imcon = 0, keyfce = 0, kmax1 = 0, kmax2 = 0, kmax3 = 0, ntpvdw = 0, mxatm = 0, mxatyp = 0;
  int maxguest = 3000, maxatm = 15000;
  double volm = 0, rcut = 0, eps = 0, alpha = 0, initdelr = 0, rvdw = 0;
  bool lcut = false, lewald = false, lrvdw = false, ldelr = false;
  double cell[9] = {0}, celprp[10] = {0};
  int mxgrid = 0, mxegrd = 0, mxebuf = 0, maxvdw = 0;
  // ---- readfield
  double engunit = 1.0;
  int ntpatm = 0, ntpmls = 0, ntpguest = 0, ntpfram = 0, totatm = 0, framatm = 0;
  std::vector<std::string> unqatm;
  std::vector<MolType> mols;
  std::vector<int> locguest, locfram;  // 0-based molecule indices
  std::vector<std::vector<double>> guestx, guesty, guestz;
  // vdw_module
  std::vector<int> ltpvdw, lstvdw;  // 1-based tables stored at [1..maxvdw]
  std::vector<std::vector<double>> prmvdw;  // [ivdw][0..4]
  std::vector<std::vector<double>> vvv;     // [ivdw][0..mxgrid]  (index 0 unused)
  std::vector<double> steadd;
  double dlrpot = 0, drewd = 0;
  std::vector<double> erc;  // [0..mxegrd]
  // ---- readcontrol
  double temp = 0;
  bool ltemp = false, lspe = false, laccsample = false, lrestart = false;
  int mcsteps = 1, eqsteps = 0, nwind = 100000;
  // numguests.out / his.xyz (readinputs.f:708-717, 860-866; gcmc.f:418-450, 785-792, 1937-1951)
  int nnumg = 1, nhis = 0;
  std::vector<FILE*> numg_f, his_f;
  // pressure equilibration (CONTROL desorb / adsorb press / adsorb guests / packing fraction /
  // finishment; readinputs.f:749-762, gcmc.f:275-281, 637-696, 1796-1808)
  int desorb = 0;
  double despre = 0, packf = 0, presleft = 0, presrate = 0;
  std::vector<double> adspres, adsguen, dqp;
  std::vector<double> gstpress, mcinsf, mcdelf, mcdisf, mcjmpf, mcflxf, mcswpf, mctraf, mcrotf, mcmjpf;
  std::vector<double> disp_ratio, tran_ratio;
  double rota_ratio = 0.5;
  // ---- condensed arrays (condense utility_pack.f:3325-3423)
  std::vector<double> xxx, yyy, zzz, atmcharge, atmweight;
  std::vector<int> ltype, lfreezesite;
  std::vector<int> nexsit;  // [iguest][site]
  std::vector<std::vector<std::vector<int>>> lexsit;
  std::vector<int> nexatm;
  std::vector<std::vector<int>> lexatm;
  std::vector<int> numtyp, numfrz;  // 1-based [1..ntpatm]
  // ---- ewald state
  std::vector<double> ckcsum, ckssum, ckcsnew, ckssnew;
  int newld = 0;
  std::vector<double> ewald3en;
  // ---- run state
  double epsq = 1.0, beta = 0, statvolm = 0, elrc = 0;
  double spenergy = 0, dlpeng = 0, ewald1sum = 0, evdwg = 0, ecoulg = 0;
  std::vector<double> energy, delE;
  std::vector<double> delr, delrdisp, tran_delr;
  std::vector<int> accept_disp, disp_count, accept_tran, tran_count;
  int accept_rota = 0, rota_count = 0, accept_ins = 0, accept_del = 0, ins_count = 0, del_count = 0;
  double rotangle = PI / 3.0, rota_rotangle = PI / 3.0;
  int gcmccount = 0;
  Duni rng;
  // production statistics (gcmc.f:1814-1860, chainstats(1+14*(i-1)+1..5))
  bool production = false;
  long long prodcount = 0;
  bool last_accepted = false;
  int jump_count = 0, accept_jump = 0;
  // windowed statistics (gcmc.f:1814-1935) and the first 500,000 production samples
  // (gasmol / gaseng) for the blocked errors of the final report (gcmc.f:1960-2037)
  int rollcount = 0, ins_rollcount = 0, avcount = 0;
  std::vector<double> avgwindow, sumwindowav, varwindow, seltot, selwin;  // [8*ng], [ng*ng]
  std::vector<double> gasmol, gaseng;                                     // [ng*500000 + 1]
  std::vector<double> chainstats;
  bool tick_tock[5] = {false, false, false, false, false};
  bool lgchk = true;
  // scratch for the per-trial neighbour list (guestlistgen)
  std::vector<int> ind;
  std::vector<double> newx, newy, newz;
  std::vector<std::vector<int>> gstlist;
  std::vector<int> gstlentry;
};

// ------------------------------------------------------------------ initscan
static void initscan(Chain& C, const std::string& dir) {
  Rec r;
  {
    LineFile f(dir + "/FIELD");
    if (!f.getrec(r)) fail(52, "end of FIELD file encountered");
    bool loop = true;
    while (loop) {
      if (!f.getrec(r)) fail(52, "end of FIELD file encountered");
      lowcase(r.c, LENREC);
      strip(r.c, LENREC);
      if (r.c[0] == '#' || r.c[0] == ' ') {
      } else if (findstring("molecu", r.c)) {
        int maxmls = intstr(r.c, LENREC, nullptr);
        std::vector<std::string> chr;
        int nummls = 0;
        for (int n = 0; n < maxmls; n++) {
          bool loop2 = true;
          while (loop2) {
            if (!f.getrec(r)) fail(52, "end of FIELD file encountered");
            lowcase(r.c, LENREC);
            strip(r.c, LENREC);
            if (r.c[0] == '#' || r.c[0] == ' ') {
            } else if (findstring("nummol", r.c)) {
              nummls = intstr(r.c, LENREC, nullptr);
            } else if (findstring("atoms", r.c)) {
              int numsit = intstr(r.c, LENREC, nullptr);
              C.mxatm += numsit * nummls;
              int ksite = 0;
              for (int isite = 0; isite < numsit; isite++) {
                if (ksite < numsit) {
                  if (!f.getrec(r)) fail(52, "end of FIELD file encountered");
                  std::string name = getword(r.c, 8, LENREC);
                  dblstr(r.c, LENREC);
                  dblstr(r.c, LENREC);
                  int nrept = intstr(r.c, LENREC, nullptr);
                  intstr(r.c, LENREC, nullptr);
                  intstr(r.c, LENREC, nullptr);
                  if (nrept == 0) nrept = 1;
                  ksite += nrept;
                  bool found = false;
                  for (auto& s : chr)
                    if (s == name) found = true;
                  if (!found) chr.push_back(name);
                }
              }
            } else if (findstring("finish", r.c)) {
              loop2 = false;
            }
          }
        }
        C.mxatyp = (int)chr.size();
      } else if (findstring("vdw", r.c)) {
        C.ntpvdw = intstr(r.c, LENREC, nullptr);
      } else if (findstring("close", r.c)) {
        loop = false;
      }
    }
  }
  {
    LineFile f(dir + "/CONFIG");
    f.getrec(r);
    f.getrec(r);
    intstr(r.c, LENREC, nullptr);
    C.imcon = intstr(r.c, LENREC, nullptr);
    for (int row = 0; row < 3; row++) {
      if (!f.getrec(r)) fail(54, "problem reading CONFIG file");
      for (int j = 0; j < 3; j++) C.cell[3 * row + j] = dblstr(r.c, LENREC);
    }
    dcell(C.cell, C.celprp);
  }
  {
    LineFile f(dir + "/CONTROL");
    bool loop3 = true;
    C.ntpguest = 0;
    while (loop3) {
      if (!f.getrec(r)) fail(53, "end of CONTROL file encountered");
      lowcase(r.c, LENREC);
      strip(r.c, LENREC);
      if (r.c[0] == '#' || r.c[0] == ' ') {
      } else if (findstring("cut", r.c)) {
        C.rcut = dblstr(r.c, LENREC);
        C.lcut = true;
      } else if (findstring("max guest atoms", r.c)) {
        C.maxguest = intstr(r.c, LENREC, nullptr);
      } else if (findstring("max framework atoms", r.c)) {
        C.maxatm = intstr(r.c, LENREC, nullptr);
      } else if (findstring("&guest", r.c)) {
        C.ntpguest++;
        bool loop4 = true;
        while (loop4) {
          if (!f.getrec(r)) fail(53, "end of CONTROL file encountered");
          lowcase(r.c, LENREC);
          strip(r.c, LENREC);
          if (r.c[0] == '#' || r.c[0] == ' ') {
          } else if (findstring("probability", r.c)) {
            int qprob = intstr(r.c, LENREC, nullptr), iprob = 0;
            while (iprob < qprob) {
              if (!f.getrec(r)) fail(53, "end of CONTROL file encountered");
              strip(r.c, LENREC);
              if (!(r.c[0] == '#' || r.c[0] == ' ')) iprob++;
            }
          } else if (findstring("&end", r.c)) {
            loop4 = false;
          }
        }
      } else if (findstring("finishment", r.c)) {
      } else if (findstring("delr", r.c)) {
        C.initdelr = dblstr(r.c, LENREC);
        C.ldelr = true;
      } else if (findstring("finish", r.c)) {
        loop3 = false;
      } else if (findstring("ewald", r.c)) {
        C.lewald = true;
        C.keyfce = 2;
        if (findstring("precision", r.c)) {
          C.eps = dblstr(r.c, LENREC);
          if (C.lcut) {
            // utility_pack.f:381-391: DL_POLY precision rule for alpha and kmax
            double eps = std::min(std::fabs(C.eps), 0.5);
            double tol = std::sqrt(std::fabs(std::log(eps * C.rcut)));
            C.alpha = std::sqrt(std::fabs(std::log(eps * C.rcut * tol))) / C.rcut;
            double tol1 = std::sqrt(-std::log(eps * C.rcut * (2.0 * tol * C.alpha) * (2.0 * tol * C.alpha)));
            double fac = 1.0;
            if (C.imcon == 4 || C.imcon == 5 || C.imcon == 7) fac = std::pow(2.0, 1.0 / 3.0);
            C.kmax1 = (int)fnint(0.25 + fac * C.celprp[0] * C.alpha * tol1 / PI);
            C.kmax2 = (int)fnint(0.25 + fac * C.celprp[1] * C.alpha * tol1 / PI);
            C.kmax3 = (int)fnint(0.25 + fac * C.celprp[2] * C.alpha * tol1 / PI);
          }
        } else {
          C.alpha = dblstr(r.c, LENREC);
          C.kmax1 = intstr(r.c, LENREC, nullptr);
          C.kmax2 = intstr(r.c, LENREC, nullptr);
          C.kmax3 = intstr(r.c, LENREC, nullptr);
        }
      } else if (findstring("rvdw", r.c)) {
        C.rvdw = dblstr(r.c, LENREC);
        C.lrvdw = true;
      } else if (findstring("grid", r.c)) {  // utility_pack.f:403-411
        if (findstring("spa", r.c)) {
          C.griddim = dblstr(r.c, LENREC);
        } else if (findstring("fac", r.c)) {
          C.gridfactor[0] = intstr(r.c, LENREC, nullptr);
          C.gridfactor[1] = intstr(r.c, LENREC, nullptr);
          C.gridfactor[2] = intstr(r.c, LENREC, nullptr);
        }
      }
    }
  }
  double width = std::min(C.celprp[6], std::min(C.celprp[7], C.celprp[8])) / 2.0;
  if (C.imcon == 4) width = std::sqrt(3.0) * C.cell[0] / 4.0;
  if (C.imcon == 5) width = C.cell[0] / 2.0;
  if (C.imcon == 6) width = std::min(C.celprp[6], C.celprp[7]) / 2.0;
  if (C.rcut > width) fail(95, "potential cutoff exceeds half-cell width");
  dcell(C.cell, C.celprp);
  if (C.imcon == 0)
    C.volm = 0.0;
  else if (C.imcon == 4 || C.imcon == 5 || C.imcon == 7)
    C.volm = 0.5 * C.celprp[9];
  else
    C.volm = C.celprp[9];
  if (!C.lrvdw && C.rcut > 0.0) C.rvdw = C.rcut;
  if (!C.lewald) fail(2311, "GCMC sim needs ewald specified in CONTROL file");
}

// loc8 utility_pack.f:2373-2389
static inline int loc8(int i, int j) {
  int a = std::max(i, j), b = std::min(i, j);
  return (a * (a - 1)) / 2 + b;
}

// forgen vdw_terms.f:189-396 (all tabulated forms)
static void forgen(Chain& C) {
  C.dlrpot = C.rvdw / (double)(C.mxgrid - 4);
  const double dl = C.dlrpot;
  for (int ivdw = 1; ivdw <= C.ntpvdw; ivdw++) {
    const double* p = C.prmvdw[ivdw].data();
    std::vector<double>& v = C.vvv[ivdw];
    int key = C.ltpvdw[ivdw];
    for (int i = 1; i <= C.mxgrid; i++) {
      double rrr = (double)i * dl;
      if (key == 1) {
        v[i] = (p[0] / powi(rrr, 6) - p[1]) / powi(rrr, 6);
      } else if (key == 2) {
        double sr = p[1] / rrr;
        v[i] = 4.0 * p[0] * powi(sr, 6) * (powi(sr, 6) - 1.0);
      } else if (key == 3) {
        double ann = std::max(p[1], p[2]), amm = std::min(p[1], p[2]);
        v[i] = p[0] / (ann - amm) * (amm * std::pow(p[3] / rrr, ann) - ann * std::pow(p[3] / rrr, amm));
      } else if (key == 4) {
        v[i] = p[0] * std::exp(-rrr / p[1]) - p[2] / powi(rrr, 6);
      } else if (key == 5) {
        v[i] = p[0] * std::exp(p[1] * (p[2] - rrr)) - p[3] / powi(rrr, 6) - p[4] / powi(rrr, 8);
      } else if (key == 6) {
        v[i] = p[0] / powi(rrr, 12) - p[1] / powi(rrr, 10);
      } else if (key == 7) {
        double eps = p[0], ann = p[1], amm = p[2], rr0 = p[3], rrc = p[4];
        if (rrc < 1e-6) rrc = C.rvdw;
        double gam = rrc / rr0;
        double bet = gam * std::pow((std::pow(gam, amm + 1.0) - 1.0) / (std::pow(gam, ann + 1.0) - 1.0),
                                    1.0 / (ann - amm));
        eps = -eps * (ann - amm) /
              (amm * std::pow(bet, ann) * (1.0 + (ann / gam - ann - 1.0) / std::pow(gam, ann)) -
               ann * std::pow(bet, amm) * (1.0 + (amm / gam - amm - 1.0) / std::pow(gam, amm)));
        if (rrr > rrc)
          v[i] = 0.0;
        else
          v[i] = eps / (ann - amm) *
                 (amm * std::pow(bet, ann) * (std::pow(rr0 / rrr, ann) - std::pow(1.0 / gam, ann)) -
                  ann * std::pow(bet, amm) * (std::pow(rr0 / rrr, amm) - std::pow(1.0 / gam, amm)) +
                  ann * amm * ((rrr / (gam * rr0) - 1.0) * (std::pow(bet / gam, ann) - std::pow(bet / gam, amm))));
      } else if (key == 8) {
        double t = 1.0 - std::exp(-p[2] * (rrr - p[1]));
        v[i] = p[0] * (t * t - 1.0);
      } else if (key == 9) {
        double eps = p[0], sig = p[1], rr0 = p[2];
        double ddd = sig * std::pow(2.0, 1.0 / 6.0);
        double rr = (double)i * dl - rr0;
        if (rr > ddd)
          v[i] = 0.0;
        else if (rr > 0.0) {
          double sr = sig / rr;
          v[i] = 4.0 * eps * powi(sr, 6) * (powi(sr, 6) - 1.0) + eps;
        }
      }
    }
  }
}

// define_van_der_waals vdw_terms.f:1-187
static void define_vdw(Chain& C, LineFile& f) {
  for (int ivdw = 1; ivdw <= C.maxvdw; ivdw++) {
    C.lstvdw[ivdw] = 0;
    C.ltpvdw[ivdw] = -1;
  }
  Rec r;
  for (int itpvdw = 1; itpvdw <= C.ntpvdw; itpvdw++) {
    double parpot[5] = {0, 0, 0, 0, 0};
    if (!f.getrec(r)) fail(52, "end of FIELD file encountered");
    std::string a1 = getword(r.c, 8, LENREC);
    std::string a2 = getword(r.c, 8, LENREC);
    lowcase(r.c, LENREC - 16);
    std::string kw = getword(r.c, 4, LENREC).substr(0, 4);
    int keypot = -1;
    if (kw == "12-6") keypot = 1;
    else if (kw == "lj  ") keypot = 2;
    else if (kw == "nm  ") keypot = 3;
    else if (kw == "buck") keypot = 4;
    else if (kw == "bhm ") keypot = 5;
    else if (kw == "hbnd") keypot = 6;
    else if (kw == "snm ") keypot = 7;
    else if (kw == "hcnm") keypot = 7;
    else if (kw == "mors") keypot = 8;
    else if (kw == "wca ") keypot = 9;
    else if (kw == "tab ") keypot = 0;
    for (int i = 0; i < 5; i++) parpot[i] = dblstr(r.c, LENREC);
    int k1 = 0, k2 = 0;
    for (int j = 1; j <= C.ntpatm; j++) {
      if (a1 == C.unqatm[j - 1]) k1 = j;
      if (a2 == C.unqatm[j - 1]) k2 = j;
    }
    if (k1 == 0 || k2 == 0) fail(4, "vdw pair names an unknown atom type");
    int keyvdw = loc8(k1, k2);
    parpot[0] *= C.engunit;
    if (keypot == 1) parpot[1] *= C.engunit;
    else if (keypot == 4) parpot[2] *= C.engunit;
    else if (keypot == 5) {
      parpot[3] *= C.engunit;
      parpot[4] *= C.engunit;
    } else if (keypot == 6)
      parpot[1] *= C.engunit;
    C.lstvdw[keyvdw] = itpvdw;
    C.ltpvdw[itpvdw] = keypot;
    for (int i = 0; i < 5; i++) C.prmvdw[itpvdw][i] = parpot[i];
  }
  if (C.ntpvdw > 0) forgen(C);
  int ntab = (C.ntpatm * (C.ntpatm + 1)) / 2;
  if (C.ntpvdw < ntab) {
    for (int i = 1; i <= ntab; i++)
      if (C.lstvdw[i] == 0) C.lstvdw[i] = C.ntpvdw + 1;
    for (int i = 0; i <= C.mxgrid; i++) C.vvv[C.ntpvdw + 1][i] = 0.0;
  }
  // The reference reads vvv(0,k) (outside its table) for pair distances below one grid step;
  // this restatement defines that entry as vvv(1,k).
  for (int k = 1; k <= C.ntpvdw + 1 && k < (int)C.vvv.size(); k++) C.vvv[k][0] = C.vvv[k][1];
}

// readfield readinputs.f:11-307
static void readfield(Chain& C, const std::string& dir) {
  LineFile f(dir + "/FIELD");
  Rec r;
  C.engunit = 1.0;
  C.totatm = 0;
  C.ntpguest = 0;
  C.ntpfram = 0;
  C.ntpatm = 0;
  C.unqatm.clear();
  C.locguest.clear();
  C.locfram.clear();
  if (!f.getrec(r)) fail(52, "end of FIELD file encountered");
  bool loop = true;
  while (loop) {
    if (!f.getrec(r)) fail(52, "end of FIELD file encountered");
    lowcase(r.c, LENREC);
    strip(r.c, LENREC);
    if (findstring("units", r.c)) {
      bool blank = true;
      for (int i = 5; i < LENREC; i++)
        if (r.c[i] != ' ') blank = false;
      if (blank) {
      } else if (findstring("ev", r.c)) C.engunit = 9648.530821;
      else if (findstring("kcal", r.c)) C.engunit = 418.4;
      else if (findstring("kj", r.c)) C.engunit = 1.0e2;
      else if (findstring("k", r.c)) C.engunit = BOLTZ;
    } else if (findstring("vdw", r.c)) {
      define_vdw(C, f);
    } else if (findstring("molecu", r.c)) {
      C.ntpmls = intstr(r.c, LENREC, nullptr);
      C.mols.assign(C.ntpmls, MolType());
      for (int n = 0; n < C.ntpmls; n++) {
        MolType& M = C.mols[n];
        if (!f.getrec(r)) fail(52, "end of FIELD file encountered");
        lowcase(r.c, LENREC);
        bool lguest = false;
        if (findstring("&guest", r.c)) {
          lguest = true;
          C.ntpguest++;
          C.locguest.push_back(n);
          C.guestx.emplace_back();
          C.guesty.emplace_back();
          C.guestz.emplace_back();
        } else {
          C.ntpfram++;
          C.locfram.push_back(n);
        }
        M.guest = lguest;
        strip(r.c, LENREC);
        M.name = std::string(r.c, 40);
        bool loop2 = true;
        while (loop2) {
          if (!f.getrec(r)) fail(52, "end of FIELD file encountered");
          lowcase(r.c, LENREC);
          strip(r.c, LENREC);
          int ksite = 0;
          if (findstring("nummol", r.c)) {
            M.nummols = intstr(r.c, LENREC, nullptr);
          } else if (findstring("atoms", r.c)) {
            int numsit = intstr(r.c, LENREC, nullptr);
            M.numatoms = numsit;
            M.atmname.assign(numsit, "");
            M.wght.assign(numsit, 0.0);
            M.chg.assign(numsit, 0.0);
            M.frz.assign(numsit, 0);
            M.ltpsit.assign(numsit, 0);
            if (lguest) {
              C.guestx.back().assign(numsit, 0.0);
              C.guesty.back().assign(numsit, 0.0);
              C.guestz.back().assign(numsit, 0.0);
            }
            for (int isite = 0; isite < numsit; isite++) {
              if (ksite < M.numatoms) {
                if (!f.getrec(r)) fail(52, "end of FIELD file encountered");
                std::string atom1 = getword(r.c, 8, LENREC);
                double weight = dblstr(r.c, LENREC);
                double charge = dblstr(r.c, LENREC);
                int nrept, ifrz;
                if (lguest) {
                  nrept = 1;
                  C.guestx.back()[isite] = dblstr(r.c, LENREC);
                  C.guesty.back()[isite] = dblstr(r.c, LENREC);
                  C.guestz.back()[isite] = dblstr(r.c, LENREC);
                  ifrz = 0;
                } else {
                  nrept = intstr(r.c, LENREC, nullptr);
                  ifrz = intstr(r.c, LENREC, nullptr);
                }
                if (nrept == 0) nrept = 1;
                for (int irept = 0; irept < nrept; irept++) {
                  if (ksite >= numsit) fail(4, "atom repeat count overruns the ATOMS block");
                  M.atmname[ksite] = atom1;
                  M.wght[ksite] = weight;
                  M.chg[ksite] = charge;
                  M.frz[ksite] = ifrz;
                  ksite++;
                }
                bool atmchk = true;
                for (int j = 1; j <= C.ntpatm; j++) {
                  if (atom1 == C.unqatm[j - 1]) {
                    atmchk = false;
                    for (int ir = ksite; ir > ksite - nrept; ir--) M.ltpsit[ir - 1] = j;
                  }
                }
                if (atmchk) {
                  C.ntpatm++;
                  C.unqatm.push_back(atom1);
                  for (int ir = ksite; ir > ksite - nrept; ir--) M.ltpsit[ir - 1] = C.ntpatm;
                }
              }
            }
          } else if (findstring("finish", r.c)) {
            loop2 = false;
            if (lguest) {
              // readinputs.f:246-268: centre the guest template on its mass COM
              double mass = 0, cx = 0, cy = 0, cz = 0;
              int g = C.ntpguest - 1;
              for (int i = 0; i < M.numatoms; i++) {
                cx = cx + C.guestx[g][i] * M.wght[i];
                cy = cy + C.guesty[g][i] * M.wght[i];
                cz = cz + C.guestz[g][i] * M.wght[i];
                mass = mass + M.wght[i];
              }
              cx = cx / mass;
              cy = cy / mass;
              cz = cz / mass;
              for (int i = 0; i < M.numatoms; i++) {
                C.guestx[g][i] -= cx;
                C.guesty[g][i] -= cy;
                C.guestz[g][i] -= cz;
              }
            }
          }
        }
        C.totatm += M.numatoms * M.nummols;
      }
    } else if (findstring("close", r.c)) {
      loop = false;
    } else {
      fail(4, "unknown directive found in FIELD file");
    }
  }
}

// Fortran '(3f20.0)' formatted read of three 20-character fields
static double ffield(const std::string& s, int k) {
  std::string t;
  for (int i = 20 * k; i < 20 * k + 20 && i < (int)s.size(); i++) {
    char ch = s[i];
    if (ch == ' ') continue;
    if (ch == 'd' || ch == 'D') ch = 'e';
    t.push_back(ch);
  }
  if (t.empty()) return 0.0;
  return std::strtod(t.c_str(), nullptr);
}

// readconfig readinputs.f:309-513
static void readconfig(Chain& C, const std::string& dir) {
  LineFile f(dir + "/CONFIG");
  Rec r;
  f.getrec(r);
  f.getrec(r);
  int levcfg = intstr(r.c, LENREC, nullptr);
  if (C.imcon == 0) {
    for (int i = 0; i < 9; i++) C.cell[i] = 0.0;
  } else {
    for (int row = 0; row < 3; row++) {
      if (!f.getrec(r)) fail(54, "problem reading CONFIG file");
      for (int j = 0; j < 3; j++) C.cell[3 * row + j] = dblstr(r.c, LENREC);
    }
  }
  for (int k = 0; k < C.ntpmls; k++) {
    MolType& M = C.mols[k];
    int n = M.nummols * M.numatoms;
    M.fx.assign(std::max(n, 1), 0.0);
    M.fy.assign(std::max(n, 1), 0.0);
    M.fz.assign(std::max(n, 1), 0.0);
    int indatm = 0;
    for (int l = 0; l < M.nummols; l++) {
      for (int m = 0; m < M.numatoms; m++) {
        std::string nl, cl, junk;
        if (!f.rawline(nl) || !f.rawline(cl)) fail(55, "end of CONFIG file encountered");
        for (int e = 0; e < levcfg; e++)
          if (!f.rawline(junk)) fail(55, "end of CONFIG file encountered");
        char an[8];
        for (int i = 0; i < 8; i++) an[i] = i < (int)nl.size() ? nl[i] : ' ';
        strip(an, 8);
        if (M.atmname[m] == std::string(an, 8)) {
          M.fx[indatm] = ffield(cl, 0);
          M.fy[indatm] = ffield(cl, 1);
          M.fz[indatm] = ffield(cl, 2);
        } else {
          fail(25, "wrong atom type found in CONFIG file");
        }
        indatm++;
      }
    }
  }
  const double* cell = C.cell;
  if (C.imcon == 1 || C.imcon == 4 || C.imcon == 5) {
    double axx = (std::fabs(cell[0]) + std::fabs(cell[4])) / 2.0, test = 1e-8 * axx;
    if (std::fabs(cell[0] - axx) > test) fail(410, "cell not consistent with image convention");
    if (std::fabs(cell[4] - axx) > test) fail(410, "cell not consistent with image convention");
    if (C.imcon == 5) {
      if (std::fabs(cell[8] - axx * std::sqrt(2.0)) > test) fail(410, "cell not consistent with image convention");
    } else if (std::fabs(cell[8] - axx) > test)
      fail(410, "cell not consistent with image convention");
  }
  if (C.imcon == 7 && std::fabs(cell[0] - std::sqrt(3.0) * cell[4]) >= 1e-6)
    fail(410, "cell not consistent with image convention");
  if (C.imcon == 6) {
    if (std::fabs(cell[2]) > 1e-10 || std::fabs(cell[5]) > 1e-10 || std::fabs(cell[6]) > 1e-10 ||
        std::fabs(cell[7]) > 1e-10)
      fail(410, "cell not consistent with image convention");
  }
  if (C.imcon == 1 || C.imcon == 2 || C.imcon == 4 || C.imcon == 5 || C.imcon == 7) {
    if (std::fabs(cell[1]) > 1e-10 || std::fabs(cell[2]) > 1e-10 || std::fabs(cell[3]) > 1e-10 ||
        std::fabs(cell[5]) > 1e-10 || std::fabs(cell[6]) > 1e-10 || std::fabs(cell[7]) > 1e-10)
      fail(410, "cell not consistent with image convention");
  }
  dcell(C.cell, C.celprp);
  if (C.imcon == 0)
    C.volm = 0.0;
  else if (C.imcon == 4 || C.imcon == 5 || C.imcon == 7)
    C.volm = 0.5 * C.celprp[9];
  else
    C.volm = C.celprp[9];
  if (C.imcon > 0) {
    double width = std::min(C.celprp[6], std::min(C.celprp[7], C.celprp[8])) / 2.0;
    if (C.imcon == 4) width = std::sqrt(3.0) * C.cell[0] / 4.0;
    if (C.imcon == 5) width = C.cell[0] / 2.0;
    if (C.imcon == 6) width = std::min(C.celprp[6], C.celprp[7]) / 2.0;
    if (C.rcut > width) fail(95, "potential cutoff exceeds half-cell width");
  }
}

// readcontrol readinputs.f:515-914 (directives that change the trajectory or the statistics)
static void readcontrol(Chain& C, const std::string& dir) {
  LineFile f(dir + "/CONTROL");
  Rec r;
  int ng = C.ntpguest;
  C.gstpress.assign(ng, 0.0);
  C.adspres.assign(ng, 0.0);
  C.adsguen.assign(ng, 0.0);
  for (auto* v : {&C.mcinsf, &C.mcdelf, &C.mcdisf, &C.mcjmpf, &C.mcflxf, &C.mcswpf, &C.mctraf, &C.mcrotf, &C.mcmjpf})
    v->assign(ng, 0.0);
  C.disp_ratio.assign(ng, 0.5);
  C.tran_ratio.assign(ng, 0.5);
  C.rota_ratio = 0.5;
  std::vector<char> mvspefid(ng, 0), disp_spefid(ng, 0), tran_spefid(ng, 0);
  bool lmcsteps = false, leqsteps = false, lwind = false, lnumg = false;
  int ngst = 0;
  if (!f.getrec(r)) fail(53, "end of CONTROL file encountered");
  bool loop = true;
  while (loop) {
    if (!f.getrec(r)) fail(53, "end of CONTROL file encountered");
    lowcase(r.c, LENREC);
    strip(r.c, LENREC);
    char* d = r.c;  // "directive" is a copy of the record
    if (d[0] == '#' || d[0] == ' ') {
    } else if (findstring("restart", d)) {
      // readinputs.f:604-608; the branch REVIVE itself is loaded by the caller (load_guests +
      // orc_restart_flags), as gcmc.f:353-418 does after the deck is read
      C.lrestart = true;
    } else if (findstring("temp", d)) {
      C.temp = dblstr(d, LENREC);
      C.ltemp = true;
    } else if (findstring("sampling", d)) {
      C.laccsample = true;
    } else if (findstring("&guest", d)) {
      ngst++;
      int idguest = intstr(d, LENREC, nullptr);
      if (idguest < 1 || idguest > ng) fail(2312, "&guest index out of range");
      int g = idguest - 1;
      Rec dir_rec = r;  // readinputs.f:686: the per-guest 'delr' test reads this outer record
      bool loop2 = true;
      while (loop2) {
        if (!f.getrec(r)) fail(53, "end of CONTROL file encountered");
        lowcase(r.c, LENREC);
        strip(r.c, LENREC);
        if (r.c[0] == '#' || r.c[0] == ' ') {
        } else if (findstring("fract", r.c)) {
          dblstr(r.c, LENREC);
        } else if (findstring("press", r.c)) {
          C.gstpress[g] = dblstr(r.c, LENREC) * 1.0e5;
        } else if (findstring("probability", r.c)) {
          int n = intstr(r.c, LENREC, nullptr), cprob = 0;
          while (cprob < n) {
            if (!f.getrec(r)) fail(53, "end of CONTROL file encountered");
            strip(r.c, LENREC);
            if (!(r.c[0] == '#' || r.c[0] == ' ')) {
              cprob++;
              ProbPlotO pl;
              pl.guest = g;
              int ns = intstr(r.c, LENREC, nullptr);
              for (int j = 0; j < ns; j++) pl.sites.push_back(intstr(r.c, LENREC, nullptr));
              C.plots.push_back(pl);
            }
          }
        } else if (findstring("move", r.c)) {
          mvspefid[g] = 1;
          if (findstring("ins", r.c)) C.mcinsf[g] = dblstr(r.c, LENREC);
          else if (findstring("del", r.c)) C.mcdelf[g] = dblstr(r.c, LENREC);
          else if (findstring("dis", r.c)) C.mcdisf[g] = dblstr(r.c, LENREC);
          else if (findstring("jum", r.c)) C.mcjmpf[g] = dblstr(r.c, LENREC);
          else if (findstring("fle", r.c)) C.mcflxf[g] = dblstr(r.c, LENREC);
          else if (findstring("swa", r.c)) C.mcswpf[g] = dblstr(r.c, LENREC);
          else if (findstring("tra", r.c)) C.mctraf[g] = dblstr(r.c, LENREC);
          else if (findstring("rot", r.c)) C.mcrotf[g] = dblstr(r.c, LENREC);
          else if (findstring("mul", r.c)) C.mcmjpf[g] = dblstr(r.c, LENREC);
        } else if (findstring("delr", dir_rec.c)) {
          dblstr(r.c, LENREC);  // dead: sets a local shadow array (readinputs.f:542,686-688)
        } else if (findstring("accep", r.c)) {
          if (findstring("dis", r.c)) {
            disp_spefid[g] = 1;
            C.disp_ratio[g] = dblstr(r.c, LENREC);
          } else if (findstring("tra", r.c)) {
            tran_spefid[g] = 1;
            C.tran_ratio[g] = dblstr(r.c, LENREC);
          }
        } else if (findstring("&end", r.c)) {
          loop2 = false;
        }
      }
    } else if (findstring("steps", d)) {
      C.mcsteps = intstr(d, LENREC, nullptr);
      lmcsteps = true;
    } else if (findstring("pressure", d) || findstring("total press", d)) {
      dblstr(d, LENREC);
    } else if (findstring("numg", d)) {
      lnumg = true;
      C.nnumg = intstr(d, LENREC, nullptr);
      if (C.nnumg <= 0) C.nnumg = 1000;
    } else if (findstring("fuga", d)) {
    } else if (findstring("hist", d)) {
      C.nhis = intstr(d, LENREC, nullptr);
    } else if (findstring("equilibr", d)) {
      C.eqsteps = intstr(d, LENREC, nullptr);
      if (C.eqsteps != 0) leqsteps = true;
    } else if (findstring("uvt", d)) {
    } else if (findstring("single point", d)) {
      C.lspe = true;
    } else if (findstring("jobcontrol", d)) {
    } else if (findstring("cutoff", d)) {
      C.rcut = dblstr(d, LENREC);
    } else if (findstring("delr", d)) {
      dblstr(d, LENREC);  // dead: local shadow array
    } else if (findstring("ewald", d)) {
    } else if (findstring("averaging window", d)) {
      C.nwind = intstr(d, LENREC, nullptr);
      lwind = true;
    } else if (findstring("max guest atoms", d)) {
      C.maxguest = intstr(d, LENREC, nullptr);
    } else if (findstring("max framework atoms", d)) {
      C.maxatm = intstr(d, LENREC, nullptr);
    } else if (findstring("desorb", d)) {
      C.desorb = intstr(d, LENREC, nullptr);
    } else if (findstring("adsorb press", d)) {
      for (int i = 0; i < ng; i++) C.adspres[i] = dblstr(d, LENREC);
    } else if (findstring("adsorb guests", d)) {
      for (int i = 0; i < ng; i++) C.adsguen[i] = dblstr(d, LENREC);
    } else if (findstring("packing fraction", d)) {
      C.packf = dblstr(d, LENREC);
    } else if (findstring("finishment", d)) {
      C.despre = dblstr(d, LENREC);
    } else if (findstring("move", d)) {
      std::vector<double>* tgt = nullptr;
      if (findstring("ins", d)) tgt = &C.mcinsf;
      else if (findstring("del", d)) tgt = &C.mcdelf;
      else if (findstring("dis", d)) tgt = &C.mcdisf;
      else if (findstring("jum", d)) tgt = &C.mcjmpf;
      else if (findstring("fle", d)) tgt = &C.mcflxf;
      else if (findstring("swa", d)) tgt = &C.mcswpf;
      else if (findstring("tra", d)) tgt = &C.mctraf;
      else if (findstring("rot", d)) tgt = &C.mcrotf;
      else if (findstring("mul", d)) tgt = &C.mcmjpf;
      if (tgt) {
        double v = dblstr(d, LENREC);
        for (int i = 0; i < ng; i++)
          if (!mvspefid[i]) (*tgt)[i] = v;
      }
    } else if (findstring("accep", d)) {
      if (findstring("dis", d)) {
        double v = dblstr(d, LENREC);
        for (int i = 0; i < ng; i++)
          if (!disp_spefid[i]) C.disp_ratio[i] = v;
      } else if (findstring("tra", d)) {
        double v = dblstr(d, LENREC);
        for (int i = 0; i < ng; i++)
          if (!tran_spefid[i]) C.tran_ratio[i] = v;
      } else if (findstring("rot", d)) {
        C.rota_ratio = dblstr(d, LENREC);
      }
    } else if (findstring("grid", d)) {
    } else if (findstring("finish", d)) {
      loop = false;
    } else {
      fail(3, "unknown directive found in CONTROL file");
    }
  }
  if (!leqsteps) C.eqsteps = 0;
  if (!lmcsteps) {
    C.mcsteps = 1;
    C.lspe = true;
  }
  if (!lwind) C.nwind = 100000;
  if (!lnumg) C.nnumg = C.eqsteps > 1000 ? C.eqsteps / 1000 : 1;
  if (C.despre > 0) {
    // the reference allocates its work array only for desorb 1, and indexes the per-guest
    // arrays by FIELD molecule index (gcmc.f:655-679), which is the guest index only when the
    // guests come first in FIELD
    if (C.desorb != 1) fail(-2, "finishment needs desorb 1");
    for (int i = 0; i < ng; i++)
      if (C.locguest[i] != i) fail(-2, "pressure equilibration needs the guests first in FIELD");
  }
  if (C.desorb == 1) C.dqp.assign(ng, 0.0);
  if (ngst != ng) fail(2312, "number of &guest blocks differs from the FIELD guests");
  if (!C.ltemp) fail(380, "simulation temperature not specified");
}

// guest_exclude utility_pack.f:3179-3263
static void guest_exclude(Chain& C) {
  C.lexsit.assign(C.ntpguest, {});
  C.nexsit.assign(C.ntpguest * 64, 0);
  for (int i = 0; i < C.ntpguest; i++) {
    int natms = C.mols[C.locguest[i]].numatoms;
    C.lexsit[i].assign(natms, std::vector<int>());
    for (int m = 0; m < natms - 1; m++) {
      for (int k = m + 1; k < natms; k++) {
        C.lexsit[i][m].push_back(k + 1);
        C.lexsit[i][k].push_back(m + 1);
      }
    }
  }
}

// condense utility_pack.f:3325-3423: guests first (by guest type), framework after
static void condense(Chain& C) {
  int total = C.totatm;
  C.xxx.assign(total, 0.0);
  C.yyy.assign(total, 0.0);
  C.zzz.assign(total, 0.0);
  C.atmcharge.assign(total, 0.0);
  C.atmweight.assign(total, 0.0);
  C.ltype.assign(total, 0);
  C.lfreezesite.assign(total, 0);
  C.nexatm.assign(total, 0);
  C.lexatm.assign(total, std::vector<int>());
  int jj = 0, lsite = 0;
  for (int g = 0; g < C.ntpguest; g++) {
    MolType& M = C.mols[C.locguest[g]];
    int ii = 0;
    for (int im = 0; im < M.nummols; im++) {
      for (int s = 0; s < M.numatoms; s++) {
        C.xxx[jj] = M.fx[ii];
        C.yyy[jj] = M.fy[ii];
        C.zzz[jj] = M.fz[ii];
        C.atmcharge[jj] = M.chg[s];
        C.lfreezesite[jj] = M.frz[s];
        C.atmweight[jj] = M.wght[s];
        C.ltype[jj] = M.ltpsit[s];
        ii++;
        jj++;  // jj is now the 1-based index of this atom
        std::vector<int>& lx = C.lexatm[jj - 1];
        for (int newsite : C.lexsit[g][s]) {
          int newatm = newsite + lsite;
          if (((newatm > jj) && (newatm - jj <= total / 2)) ||
              ((newatm < jj) && (newatm + total - jj <= (total - 1) / 2))) {
            lx.push_back(newatm);
            for (int j = (int)lx.size() - 1; j >= 1; j--)
              if (lx[j] < lx[j - 1]) std::swap(lx[j], lx[j - 1]);
          }
        }
        C.nexatm[jj - 1] = (int)lx.size();
      }
      lsite += M.numatoms;
    }
  }
  for (int t = 0; t < C.ntpfram; t++) {
    MolType& M = C.mols[C.locfram[t]];
    int ii = 0;
    for (int im = 0; im < M.nummols; im++) {
      for (int k = 0; k < M.numatoms; k++) {
        C.xxx[jj] = M.fx[ii];
        C.yyy[jj] = M.fy[ii];
        C.zzz[jj] = M.fz[ii];
        C.atmcharge[jj] = M.chg[k];
        C.lfreezesite[jj] = M.frz[k];
        C.atmweight[jj] = M.wght[k];
        C.ltype[jj] = M.ltpsit[k];
        jj++;
        ii++;
      }
    }
  }
}

// erfcgen ewald.f:1-30 (A&S 7.1.26 erfc(alpha r)/r on the grid r_i = i*drewd)
static void erfcgen(Chain& C) {
  const double a1 = 0.254829592, a2 = -0.284496736, a3 = 1.421413741;
  const double a4 = -1.453152027, a5 = 1.061405429, pp = 0.3275911;
  C.erc.assign(C.mxegrd + 1, 0.0);
  if (C.keyfce / 2 == 1 || C.keyfce / 2 == 6) {
    C.drewd = C.rcut / (double)(C.mxegrd - 4);
    for (int i = 1; i <= C.mxegrd; i++) {
      double rrr = (double)i * C.drewd;
      double tt = 1.0 / (1.0 + pp * C.alpha * rrr);
      double ar = C.alpha * rrr;
      double exp1 = std::exp(-(ar * ar));
      C.erc[i] = tt * (a1 + tt * (a2 + tt * (a3 + tt * (a4 + tt * a5)))) * exp1 / rrr;
    }
  }
  // The reference reads erc(0) (out of its table) for pair distances below one grid step;
  // this restatement defines that entry as erc(1).
  C.erc[0] = C.erc[1];
}

// Phase tables of one set of sites: e^{i 2 pi l s} for l = 0..kmax per axis (ewald.f:95-137).
struct Phases {
  int n = 0, k1 = 0, k2 = 0, k3 = 0;
  std::vector<double> elc0, els0, elc1, els1, emc, ems, enc, ens;  // emc[i*(k2+1)+l]
};
static void build_phases(Phases& P, const double* rc, int n, const double* x, const double* y, const double* z,
                         int k1, int k2, int k3) {
  const double twopi = 2.0 * PI;
  P.n = n;
  P.k1 = k1;
  P.k2 = k2;
  P.k3 = k3;
  P.elc0.assign(n, 1.0);
  P.els0.assign(n, 0.0);
  P.elc1.assign(n, 0.0);
  P.els1.assign(n, 0.0);
  P.emc.assign(n * (k2 + 1), 0.0);
  P.ems.assign(n * (k2 + 1), 0.0);
  P.enc.assign(n * (k3 + 1), 0.0);
  P.ens.assign(n * (k3 + 1), 0.0);
  for (int i = 0; i < n; i++) {
    double ssx = rc[0] * x[i] + rc[3] * y[i] + rc[6] * z[i];
    double ssy = rc[1] * x[i] + rc[4] * y[i] + rc[7] * z[i];
    double ssz = rc[2] * x[i] + rc[5] * y[i] + rc[8] * z[i];
    P.emc[i * (k2 + 1)] = 1.0;
    P.ems[i * (k2 + 1)] = 0.0;
    P.enc[i * (k3 + 1)] = 1.0;
    P.ens[i * (k3 + 1)] = 0.0;
    P.elc1[i] = std::cos(twopi * ssx);
    if (k2 >= 1) P.emc[i * (k2 + 1) + 1] = std::cos(twopi * ssy);
    if (k3 >= 1) P.enc[i * (k3 + 1) + 1] = std::cos(twopi * ssz);
    P.els1[i] = std::sin(twopi * ssx);
    if (k2 >= 1) P.ems[i * (k2 + 1) + 1] = std::sin(twopi * ssy);
    if (k3 >= 1) P.ens[i * (k3 + 1) + 1] = std::sin(twopi * ssz);
  }
  for (int l = 2; l <= k2; l++)
    for (int i = 0; i < n; i++) {
      int b = i * (k2 + 1);
      P.emc[b + l] = P.emc[b + l - 1] * P.emc[b + 1] - P.ems[b + l - 1] * P.ems[b + 1];
      P.ems[b + l] = P.ems[b + l - 1] * P.emc[b + 1] + P.emc[b + l - 1] * P.ems[b + 1];
    }
  for (int l = 2; l <= k3; l++)
    for (int i = 0; i < n; i++) {
      int b = i * (k3 + 1);
      P.enc[b + l] = P.enc[b + l - 1] * P.enc[b + 1] - P.ens[b + l - 1] * P.ens[b + 1];
      P.ens[b + l] = P.ens[b + l - 1] * P.enc[b + 1] + P.enc[b + l - 1] * P.ens[b + 1];
    }
}

// The common reciprocal-space walk of ewald1 (ewald.f:368-630) and ewald1_guest (ewald.f:32-365):
// visits every k = (l,m,n) of the reference's half-space enumeration inside rcpct2 in the
// reference's order and hands (kkk, rksq, ckcs, ckss) to the visitor.
template <class F>
static void recip_walk(Chain& C, const double* x, const double* y, const double* z, const double* q, int n,
                       F&& visit) {
  const double twopi = 2.0 * PI;
  double rc[9], det, buf[10];
  invert(C.cell, rc, &det);
  dcell(rc, buf);
  double rcpcut = std::min(std::min((double)C.kmax1 * buf[6], (double)C.kmax2 * buf[7]), (double)C.kmax3 * buf[8]);
  rcpcut = rcpcut * 1.05 * twopi;
  double rcpct2 = rcpcut * rcpcut;
  Phases P;
  build_phases(P, rc, n, x, y, z, C.kmax1, C.kmax2, C.kmax3);
  std::vector<double> clm(n), slm(n), ckc(n), cks(n);
  const int k2 = C.kmax2, k3 = C.kmax3;
  int kkk = 0, mmin = 0, nmin = 1;
  for (int ll = 0; ll <= C.kmax1; ll++) {
    int l = ll;
    double tmp = twopi * (double)ll;
    double rkx1 = tmp * rc[0], rky1 = tmp * rc[3], rkz1 = tmp * rc[6];
    if (l == 1) {
      for (int i = 0; i < n; i++) {
        P.elc0[i] = P.elc1[i];
        P.els0[i] = P.els1[i];
      }
    } else if (l > 1) {
      for (int i = 0; i < n; i++) {
        double cs = P.elc0[i];
        P.elc0[i] = cs * P.elc1[i] - P.els0[i] * P.els1[i];
        P.els0[i] = P.els0[i] * P.elc1[i] + cs * P.els1[i];
      }
    }
    for (int mm = mmin; mm <= k2; mm++) {
      int m = std::abs(mm);
      double tmp2 = twopi * (double)mm;
      double rkx2 = rkx1 + tmp2 * rc[1], rky2 = rky1 + tmp2 * rc[4], rkz2 = rkz1 + tmp2 * rc[7];
      if (mm >= 0) {
        for (int i = 0; i < n; i++) {
          double ec = P.emc[i * (k2 + 1) + m], es = P.ems[i * (k2 + 1) + m];
          clm[i] = P.elc0[i] * ec - P.els0[i] * es;
          slm[i] = P.els0[i] * ec + es * P.elc0[i];
        }
      } else {
        for (int i = 0; i < n; i++) {
          double ec = P.emc[i * (k2 + 1) + m], es = P.ems[i * (k2 + 1) + m];
          clm[i] = P.elc0[i] * ec + P.els0[i] * es;
          slm[i] = P.els0[i] * ec - es * P.elc0[i];
        }
      }
      for (int nn = nmin; nn <= k3; nn++) {
        int nabs = std::abs(nn);
        double tmp3 = twopi * (double)nn;
        double rkx3 = rkx2 + tmp3 * rc[2], rky3 = rky2 + tmp3 * rc[5], rkz3 = rkz2 + tmp3 * rc[8];
        double rksq = rkx3 * rkx3 + rky3 * rky3 + rkz3 * rkz3;
        if (rksq <= rcpct2) {
          if (nn >= 0) {
            for (int i = 0; i < n; i++) {
              double tc = P.enc[i * (k3 + 1) + nabs], ts = P.ens[i * (k3 + 1) + nabs];
              ckc[i] = q[i] * (clm[i] * tc - slm[i] * ts);
              cks[i] = q[i] * (slm[i] * tc + clm[i] * ts);
            }
          } else {
            for (int i = 0; i < n; i++) {
              double tc = P.enc[i * (k3 + 1) + nabs], ts = P.ens[i * (k3 + 1) + nabs];
              ckc[i] = q[i] * (clm[i] * tc + slm[i] * ts);
              cks[i] = q[i] * (slm[i] * tc - clm[i] * ts);
            }
          }
          double ckcs = 0.0, ckss = 0.0;
          for (int i = 0; i < n; i++) {
            ckcs = ckcs + ckc[i];
            ckss = ckss + cks[i];
          }
          visit(kkk, ll, mm, nn, rksq, ckcs, ckss);
          kkk++;
        }
      }
      nmin = -k3;
    }
    mmin = -k2;
  }
}

static bool lconsw_of(int imcon) { return !(imcon == 4 || imcon == 5 || imcon == 7); }

// ewald1 ewald.f:368-630: full S(k) of the first `natm` condensed atoms; E_recip + E_self
static double ewald1(Chain& C, int natm, double* engsic_out) {
  const double twopi = 2.0 * PI;
  double rvolm = twopi / C.volm, ralph = -0.25 / (C.alpha * C.alpha);
  bool lconsw = lconsw_of(C.imcon);
  if (!lconsw) rvolm = 0.5 * rvolm;
  double engsic = 0.0;
  for (int i = 0; i < natm; i++) engsic = engsic + C.atmcharge[i] * C.atmcharge[i];
  engsic = -R4PIE0 / C.epsq * C.alpha * engsic / SQRPI;
  double engcpe = 0.0;
  recip_walk(C, C.xxx.data(), C.yyy.data(), C.zzz.data(), C.atmcharge.data(), natm,
             [&](int kkk, int, int, int, double rksq, double ckcs, double ckss) {
               C.ckcsum[kkk] = ckcs;
               C.ckssum[kkk] = ckss;
               double rrksq = 1.0 / rksq;
               double akk = lconsw ? std::exp(ralph * rksq) * rrksq : 4.0 * std::exp(ralph * rksq) * rrksq;
               engcpe = engcpe + akk * (ckcs * ckcs + ckss * ckss);
               C.newld = kkk + 1;
             });
  if (engsic_out) *engsic_out = engsic;
  if (lconsw)
    return 2.0 * rvolm * R4PIE0 * engcpe / C.epsq + engsic;
  return rvolm * R4PIE0 * engcpe / C.epsq + engsic;
}

enum { MV_INSERT = 1, MV_DELETE = 2, MV_DISPLACE = 3 };

// ewald1_guest ewald.f:32-365 for one pass of one guest (sites newx/newy/newz)
static double ewald1_guest(Chain& C, int iguest, int natms, const double* x, const double* y, const double* z,
                           int move, int pass) {
  const double twopi = 2.0 * PI;
  const MolType& M = C.mols[C.locguest[iguest]];
  double rvolm = twopi / C.volm, ralph = -0.25 / (C.alpha * C.alpha);
  bool lconsw = lconsw_of(C.imcon);
  if (!lconsw) rvolm = 0.5 * rvolm;
  double engsic = 0.0;
  for (int i = 0; i < natms; i++) engsic = engsic + M.chg[i] * M.chg[i];
  engsic = -R4PIE0 / C.epsq * C.alpha * engsic / SQRPI;
  double engcpe = 0.0;
  recip_walk(C, x, y, z, M.chg.data(), natms, [&](int kkk, int, int, int, double rksq, double ckcs, double ckss) {
    double ckcold = C.ckcsum[kkk], cksold = C.ckssum[kkk];
    if (move == MV_INSERT) {
      ckcs = ckcs + ckcold;
      ckss = ckss + cksold;
      C.ckcsnew[kkk] = ckcs;
      C.ckssnew[kkk] = ckss;
    } else if (move == MV_DELETE) {
      ckcs = ckcold - ckcs;
      ckss = cksold - ckss;
      C.ckcsnew[kkk] = ckcs;
      C.ckssnew[kkk] = ckss;
    } else {
      if (pass == 1) {
        C.ckcsnew[kkk] = ckcold - ckcs;
        C.ckssnew[kkk] = cksold - ckss;
      } else {
        ckcs = C.ckcsnew[kkk] + ckcs;
        ckss = C.ckssnew[kkk] + ckss;
        C.ckcsnew[kkk] = ckcs;
        C.ckssnew[kkk] = ckss;
      }
    }
    double rrksq = 1.0 / rksq;
    double akk = lconsw ? std::exp(ralph * rksq) * rrksq : 4.0 * std::exp(ralph * rksq) * rrksq;
    if (move == MV_DISPLACE) {
      if (pass == 2) engcpe = engcpe + akk * (ckcs * ckcs + ckss * ckss - ckcold * ckcold - cksold * cksold);
    } else {
      engcpe = engcpe + akk * (ckcs * ckcs + ckss * ckss - ckcold * ckcold - cksold * cksold);
    }
  });
  double pref = lconsw ? 2.0 * rvolm : rvolm;
  if (move == MV_DISPLACE) return pref * R4PIE0 * engcpe / C.epsq;
  if (move == MV_DELETE) return pref * R4PIE0 * engcpe / C.epsq - engsic;
  return pref * R4PIE0 * engcpe / C.epsq + engsic;
}

// ewald2 ewald.f:632-694 over a gathered list (ilist, rsqdf)
static double ewald2(const Chain& C, double chg, int natm, const int* ilist, const double* rsqdf) {
  double rcsq = C.rcut * C.rcut, rdrewd = 1.0 / C.drewd, eng = 0.0;
  double chgea = chg / C.epsq * R4PIE0;
  for (int i = 0; i < natm; i++) {
    int jatm = ilist[i];
    double chgprd = chgea * C.atmcharge[jatm];
    if (std::fabs(chgprd) > 1e-10) {
      double rsq = rsqdf[i];
      if (rcsq > rsq) {
        double rrr = std::sqrt(rsq);
        int ll = (int)(rrr * rdrewd);
        double ppp = rrr * rdrewd - (double)ll;
        double vk0 = C.erc[ll], vk1 = C.erc[ll + 1], vk2 = C.erc[ll + 2];
        double t1 = vk0 + (vk1 - vk0) * ppp;
        double t2 = vk1 + (vk2 - vk1) * (ppp - 1.0);
        eng = eng + (t1 + (t2 - t1) * ppp * 0.5) * chgprd;
      }
    }
  }
  return eng;
}

// srfrce vdw_terms.f:398-498 over a gathered list
static double srfrce(const Chain& C, int sittyp, int ik, const int* ilist, const double* rsqdf) {
  double rcsq = C.rcut * C.rcut, rdr = 1.0 / C.dlrpot, eng = 0.0;
  double ai = (double)sittyp;
  for (int m = 0; m < ik; m++) {
    int jatm = ilist[m];
    double aj = (double)C.ltype[jatm], ab;
    if (ai > aj)
      ab = ai * (ai - 1.0) * 0.5 + aj + 0.5;
    else
      ab = aj * (aj - 1.0) * 0.5 + ai + 0.5;
    int k = C.lstvdw[(int)ab];
    if ((C.ltpvdw[k] < 100) && (std::fabs(C.vvv[k][1]) > 1e-10)) {
      double rsq = rsqdf[m];
      if (rcsq > rsq) {
        double rrr = std::sqrt(rsq);
        int l = (int)(rrr * rdr);
        double ppp = rrr * rdr - (double)l;
        const std::vector<double>& v = C.vvv[k];
        double vk0 = v[l], vk1 = v[l + 1], vk2 = v[l + 2];
        double t1 = vk0 + (vk1 - vk0) * ppp;
        double t2 = vk1 + (vk2 - vk1) * (ppp - 1.0);
        eng = (t1 + (t2 - t1) * ppp * 0.5) + eng;
      }
    }
  }
  return eng;
}

// ewald3 ewald.f:697-758 (intramolecular exclusion correction); q of partner via qj()
template <class QJ>
static double ewald3(const Chain& C, double chg, int n, const double* xdf, const double* ydf, const double* zdf,
                     QJ&& qj) {
  const double a1 = 0.254829592, a2 = -0.284496736, a3 = 1.421413741;
  const double a4 = -1.453152027, a5 = 1.061405429, pp = 0.3275911;
  const double rr3 = 0.333333333333, r10 = 0.1, r42 = 0.02380952381, r216 = 4.62962962963e-3;
  double eng = 0.0, chgea = chg / C.epsq * R4PIE0, alpha = C.alpha;
  for (int m = 0; m < n; m++) {
    double chgprd = chgea * qj(m);
    double rsq = xdf[m] * xdf[m] + ydf[m] * ydf[m] + zdf[m] * zdf[m];
    double rrr = std::sqrt(rsq), alpr = rrr * alpha, alpr2 = alpr * alpr, erfr;
    if (alpr < 1e-2) {
      erfr = 2.0 * chgprd * (alpha / SQRPI) * (1.0 + alpr2 * (-rr3 + alpr2 * (r10 + alpr2 * (-r42 + alpr2 * r216))));
    } else {
      double tt = 1.0 / (1.0 + pp * alpha * rrr);
      double ar = alpha * rrr;
      double exp1 = std::exp(-(ar * ar));
      erfr = (1.0 - tt * (a1 + tt * (a2 + tt * (a3 + tt * (a4 + tt * a5)))) * exp1) * chgprd / rrr;
    }
    eng = eng - erfr;
  }
  return eng;
}

// lrcorrect vdw_terms.f:500-682 (energy part); also fills steadd and numtyp/numfrz
static double lrcorrect(Chain& C, int natms) {
  const double twopi = 2.0 * PI;
  C.numtyp.assign(C.ntpatm + 1, 0);
  C.numfrz.assign(C.ntpatm + 1, 0);
  for (int i = 0; i < natms; i++) {
    int ka = C.ltype[i];
    C.numtyp[ka]++;
    if (C.lfreezesite[i] != 0) C.numfrz[ka]++;
  }
  double elrc = 0.0, rcut = C.rcut, volm = C.volm;
  if (C.imcon != 0 && C.imcon != 6 && C.maxvdw > 0 && C.keyfce % 2 == 0) {
    int ivdw = 0;
    for (int i = 1; i <= C.ntpatm; i++) {
      for (int j = 1; j <= i; j++) {
        double eadd = 0.0;
        ivdw++;
        int k = C.lstvdw[ivdw];
        const double* p = C.prmvdw[k].data();
        int key = C.ltpvdw[k];
        if (key == 0) {
          eadd = p[0];
        } else if (key == 1) {
          eadd = p[0] / (9.0 * powi(rcut, 9)) - p[1] / (3.0 * powi(rcut, 3));
        } else if (key == 2) {
          eadd = 4.0 * p[0] * (powi(p[1], 12) / (9.0 * powi(rcut, 9)) - powi(p[1], 6) / (3.0 * powi(rcut, 3)));
        } else if (key == 3) {
          double eps = p[0], ann = p[1], amm = p[2], rr0 = p[3];
          eadd = eps / (ann - amm) *
                 (amm * std::pow(rr0, ann) / ((ann - 3.0) * std::pow(rcut, ann - 3.0)) -
                  ann * std::pow(rr0, amm) / ((amm - 3.0) * std::pow(rcut, amm - 3.0)));
        } else if (key == 4) {
          eadd = -p[2] / (3.0 * powi(rcut, 3));
        } else if (key == 5) {
          eadd = -p[3] / (3.0 * powi(rcut, 3)) - p[4] / (5.0 * powi(rcut, 5));
        } else if (key == 6) {
          eadd = p[0] / (9.0 * powi(rcut, 9)) - p[1] / (7.0 * powi(rcut, 7));
        }
        if (i != j) eadd = eadd * 2.0;
        C.steadd[ivdw] = eadd;
        double denprd = twopi * ((double)C.numtyp[i] * (double)C.numtyp[j] - (double)C.numfrz[i] * (double)C.numfrz[j]) /
                        (volm * volm);
        elrc = elrc + volm * denprd * eadd;
      }
    }
  }
  return elrc;
}

// gstlrcorrect vdw_terms.f:684-745
static double gstlrcorrect(const Chain& C) {
  const double twopi = 2.0 * PI;
  double delrc = 0.0, volm = C.volm;
  if (C.imcon != 0 && C.imcon != 6 && C.maxvdw > 0 && C.keyfce % 2 == 0) {
    int ivdw = 0;
    for (int i = 1; i <= C.ntpatm; i++)
      for (int j = 1; j <= i; j++) {
        ivdw++;
        double eadd = C.steadd[ivdw];
        double denprd = twopi * ((double)C.numtyp[i] * (double)C.numtyp[j] - (double)C.numfrz[i] * (double)C.numfrz[j]) /
                        (volm * volm);
        delrc = delrc + volm * denprd * eadd;
      }
  }
  return delrc;
}

// guestlistgen utility_pack.f:3113-3177 + the gather of gcmc.f:906-919, then ewald2 and srfrce
// for every site; returns ewald2 and vdw sums (each site added in order).  ind[] holds the
// 0-based condensed indices of the moving molecule (-1: none).
static void guest_realspace(Chain& C, int natms, const double* nx, const double* ny, const double* nz,
                            const int* ind, const double* chg, const int* sittyp, double* ewld2sum, double* vdwsum,
                            double* site_e2 = nullptr, double* site_vdw = nullptr) {
  int total = C.totatm;
  double rclim = (C.rcut + C.delr[0]) * (C.rcut + C.delr[0]);
  std::vector<double> xdf(total), ydf(total), zdf(total), rsqdf(total);
  std::vector<int> list(total);
  *ewld2sum = 0.0;
  *vdwsum = 0.0;
  for (int i = 0; i < natms; i++) {
    int ii = 0;
    for (int j = 0; j < total; j++) {
      bool chk = true;
      for (int t = 0; t < natms; t++)
        if (j == ind[t]) chk = false;
      if (chk) {
        xdf[ii] = nx[i] - C.xxx[j];
        ydf[ii] = ny[i] - C.yyy[j];
        zdf[ii] = nz[i] - C.zzz[j];
        ii++;
      }
    }
    images(C.imcon, ii, C.cell, xdf.data(), ydf.data(), zdf.data());
    int ent = 0;
    ii = 0;
    for (int j = 0; j < total; j++) {
      bool chk = true;
      for (int t = 0; t < natms; t++)
        if (j == ind[t]) chk = false;
      if (chk) {
        double rsq;
        if (C.imcon == 6)
          rsq = xdf[ii] * xdf[ii] + ydf[ii] * ydf[ii];
        else
          rsq = xdf[ii] * xdf[ii] + ydf[ii] * ydf[ii] + zdf[ii] * zdf[ii];
        if (rsq <= rclim) list[ent++] = j;
        ii++;
      }
    }
    // gather (gcmc.f:906-919): recompute separations of the listed atoms and image them
    for (int j = 0; j < ent; j++) {
      int jatm = list[j];
      xdf[j] = nx[i] - C.xxx[jatm];
      ydf[j] = ny[i] - C.yyy[jatm];
      zdf[j] = nz[i] - C.zzz[jatm];
    }
    images(C.imcon, ent, C.cell, xdf.data(), ydf.data(), zdf.data());
    for (int l = 0; l < ent; l++) rsqdf[l] = xdf[l] * xdf[l] + ydf[l] * ydf[l] + zdf[l] * zdf[l];
    double e2 = ewald2(C, chg[i], ent, list.data(), rsqdf.data());
    double ev = srfrce(C, sittyp[i], ent, list.data(), rsqdf.data());
    if (site_e2) site_e2[i] = e2;
    if (site_vdw) site_vdw[i] = ev;
    *ewld2sum += e2;
    *vdwsum += ev;
  }
}

// parlst nlist_builders.f:1-194 (Brode-Ahlrichs Verlet list) followed by the single-point
// guest energies of gcmc.f:2639-2702.
static void single_point(Chain& C) {
  double elrc = lrcorrect(C, C.totatm);  // single_point's own local elrc (gcmc.f:2550)
  erfcgen(C);
  // condensefram + framework-only ewald1 (gcmc.f:2555-2562): framework atoms only
  {
    Chain F = C;  // a framework-only condensed view
    int jj = 0;
    int nf = 0;
    for (int t = 0; t < C.ntpfram; t++) nf += C.mols[C.locfram[t]].nummols * C.mols[C.locfram[t]].numatoms;
    F.xxx.assign(nf, 0.0);
    F.yyy.assign(nf, 0.0);
    F.zzz.assign(nf, 0.0);
    F.atmcharge.assign(nf, 0.0);
    for (int t = 0; t < C.ntpfram; t++) {
      const MolType& M = C.mols[C.locfram[t]];
      int ii = 0;
      for (int im = 0; im < M.nummols; im++)
        for (int k = 0; k < M.numatoms; k++) {
          F.xxx[jj] = M.fx[ii];
          F.yyy[jj] = M.fy[ii];
          F.zzz[jj] = M.fz[ii];
          F.atmcharge[jj] = M.chg[k];
          jj++;
          ii++;
        }
    }
    C.ewald1sum = ewald1(F, nf, nullptr);
  }
  condense(C);
  double engcpe = ewald1(C, C.totatm, nullptr);
  double ewald1eng = engcpe - C.ewald1sum;
  double ewald2eng = 0, vdweng = 0, ewald3eng = 0;
  int totfram = 0;
  for (int t = 0; t < C.ntpfram; t++) totfram += C.mols[C.locfram[t]].nummols * C.mols[C.locfram[t]].numatoms;
  if (C.totatm > totfram) {
    int natms = C.totatm;
    int last = natms, mpm2 = natms / 2, npm2 = (natms - 1) / 2;
    double rclim = (C.rcut + C.delr[0]) * (C.rcut + C.delr[0]);
    std::vector<std::vector<int>> list(natms);
    std::vector<int> noxatm(natms, 1);
    std::vector<double> xdf(natms), ydf(natms), zdf(natms);
    for (int m = 1; m <= mpm2; m++) {
      if (m > npm2) last = mpm2;
      int ii = 0;
      for (int i = 1; i <= last; i++) {
        int j = i + m;
        if (j > natms) j = j - natms;
        xdf[ii] = C.xxx[i - 1] - C.xxx[j - 1];
        ydf[ii] = C.yyy[i - 1] - C.yyy[j - 1];
        zdf[ii] = C.zzz[i - 1] - C.zzz[j - 1];
        ii++;
      }
      images(C.imcon, ii, C.cell, xdf.data(), ydf.data(), zdf.data());
      ii = 0;
      for (int i = 1; i <= last; i++) {
        bool lfrzi = C.lfreezesite[i - 1] != 0;
        int j = i + m;
        if (j > natms) j = j - natms;
        ii++;
        int a = ii - 1;
        if (C.nexatm[a] > 0 && C.lexatm[a][noxatm[a] - 1] == j) {
          noxatm[a] = std::min(noxatm[a] + 1, C.nexatm[a]);
        } else {
          bool ldo = true;
          if (lfrzi) ldo = (C.lfreezesite[j - 1] == 0);
          if (ldo) {
            double rsq = C.imcon == 6 ? xdf[a] * xdf[a] + ydf[a] * ydf[a]
                                      : xdf[a] * xdf[a] + ydf[a] * ydf[a] + zdf[a] * zdf[a];
            if (rsq < rclim && rsq >= 0.0) list[a].push_back(j - 1);
          }
        }
      }
    }
    std::vector<double> rsqdf(natms);
    for (int i = 0; i < natms; i++) {
      int n = (int)list[i].size();
      for (int k = 0; k < n; k++) {
        int j = list[i][k];
        xdf[k] = C.xxx[i] - C.xxx[j];
        ydf[k] = C.yyy[i] - C.yyy[j];
        zdf[k] = C.zzz[i] - C.zzz[j];
      }
      images(C.imcon, n, C.cell, xdf.data(), ydf.data(), zdf.data());
      for (int k = 0; k < n; k++) rsqdf[k] = xdf[k] * xdf[k] + ydf[k] * ydf[k] + zdf[k] * zdf[k];
      ewald2eng += ewald2(C, C.atmcharge[i], n, list[i].data(), rsqdf.data());
      vdweng += srfrce(C, C.ltype[i], n, list[i].data(), rsqdf.data());
    }
    for (int i = 0; i < natms; i++) {
      int n = C.nexatm[i];
      for (int k = 0; k < n; k++) {
        int j = C.lexatm[i][k] - 1;
        xdf[k] = C.xxx[i] - C.xxx[j];
        ydf[k] = C.yyy[i] - C.yyy[j];
        zdf[k] = C.zzz[i] - C.zzz[j];
      }
      images(C.imcon, n, C.cell, xdf.data(), ydf.data(), zdf.data());
      ewald3eng += ewald3(C, C.atmcharge[i], n, xdf.data(), ydf.data(), zdf.data(),
                          [&](int k) { return C.atmcharge[C.lexatm[i][k] - 1]; });
    }
    C.ecoulg = ewald1eng + ewald2eng + ewald3eng;
    C.evdwg = vdweng + elrc;
  }
  C.spenergy = (C.ecoulg + C.evdwg) / C.engunit;
  C.dlpeng = (ewald1eng + C.ewald1sum + ewald2eng + vdweng + elrc + ewald3eng) / C.engunit;
}

// ---------------------------------------------------------------- trial generators
static void cartesian(const Chain& C, double a, double b, double c, double* x, double* y, double* z) {
  *x = a * C.cell[0] + b * C.cell[3] + c * C.cell[6];
  *y = a * C.cell[1] + b * C.cell[4] + c * C.cell[7];
  *z = a * C.cell[2] + b * C.cell[5] + c * C.cell[8];
}
// rotation utility_pack.f:2887-2926
static void rotation(double* x, double* y, double* z, int n, double q1, double q2, double q3, double q4) {
  double Q[9];
  Q[0] = 2.0 * q2 * q2 + 2.0 * q1 * q1 - 1.0;
  Q[1] = 2.0 * q2 * q3 - 2.0 * q1 * q4;
  Q[2] = 2.0 * q2 * q4 + 2.0 * q1 * q3;
  Q[3] = 2.0 * q2 * q3 + 2.0 * q1 * q4;
  Q[4] = 2.0 * q1 * q1 + 2.0 * q3 * q3 - 1.0;
  Q[5] = 2.0 * q3 * q4 - 2.0 * q1 * q2;
  Q[6] = 2.0 * q2 * q4 - 2.0 * q1 * q3;
  Q[7] = 2.0 * q3 * q4 + 2.0 * q1 * q2;
  Q[8] = 2.0 * q4 * q4 + 2.0 * q1 * q1 - 1.0;
  for (int i = 0; i < n; i++) {
    double tx = Q[0] * x[i] + Q[1] * y[i] + Q[2] * z[i];
    double ty = Q[3] * x[i] + Q[4] * y[i] + Q[5] * z[i];
    double tz = Q[6] * x[i] + Q[7] * y[i] + Q[8] * z[i];
    x[i] = tx;
    y[i] = ty;
    z[i] = tz;
  }
}
static void quat_from(double theta, double r2, double r3, double r4, double* q) {
  double b1 = 2.0 * r2 - 1.0, b2 = 2.0 * r3 - 1.0, b3 = 2.0 * r4 - 1.0;
  double st = std::sin(theta / 2.0);
  double norm = std::sqrt(b1 * b1 + b2 * b2 + b3 * b3);
  double u1 = b1 / norm, u2 = b2 / norm, u3 = b3 / norm;
  q[0] = std::cos(theta / 2.0);
  q[1] = st * u1;
  q[2] = st * u2;
  q[3] = st * u3;
}
// random_ins utility_pack.f:2545-2650
static void random_ins(Chain& C, int iguest, int natms, double ra, double rb, double rcc, double r1, double r2,
                       double r3, double r4) {
  double xc, yc, zc;
  cartesian(C, ra, rb, rcc, &xc, &yc, &zc);
  for (int i = 0; i < natms; i++) {
    C.newx[i] = C.guestx[iguest][i];
    C.newy[i] = C.guesty[iguest][i];
    C.newz[i] = C.guestz[iguest][i];
  }
  double theta = r1 * 2.0 * PI, q[4];
  quat_from(theta, r2, r3, r4, q);
  rotation(C.newx.data(), C.newy.data(), C.newz.data(), natms, q[0], q[1], q[2], q[3]);
  for (int i = 0; i < natms; i++) {
    C.newx[i] = C.newx[i] + xc;
    C.newy[i] = C.newy[i] + yc;
    C.newz[i] = C.newz[i] + zc;
  }
}
// com utility_pack.f:3003-3034
static void com(const MolType& M, int natms, const double* x, const double* y, const double* z, double* cx,
                double* cy, double* cz) {
  double w = 0, sx = 0, sy = 0, sz = 0;
  for (int i = 0; i < natms; i++) {
    double mass = M.wght[i];
    w = w + mass;
    sx = sx + x[i] * mass;
    sy = sy + y[i] * mass;
    sz = sz + z[i] * mass;
  }
  *cx = sx / w;
  *cy = sy / w;
  *cz = sz / w;
}
// equitable_bin (utility_pack.f:1880-1990): the unit weight of fractional position (fa, fb, fc)
// spread over the 8 grid cells around it, linear in each direction between cell centres.
static void equitable_axis(int n, double f, int* lo, int* hi, double* wl, double* wr) {
  double gp = n * f;
  int idx = (int)std::ceil(gp);
  double part = gp - std::floor(gp);
  if (part > 0.5) {
    if (idx >= n) {
      *lo = n - 1;
      *hi = 0;
    } else {
      *lo = idx - 1;
      *hi = idx;
    }
    *wl = 1.5 - part;
    *wr = part - 0.5;
  } else {
    if (idx <= 1) {
      *lo = n - 1;
      *hi = 0;
    } else {
      *lo = idx - 2;
      *hi = idx - 1;
    }
    *wl = 0.5 - part;
    *wr = 0.5 + part;
  }
}
static void equitable_bin(Chain& C, double fa, double fb, double fc, std::vector<double>& g) {
  const int na = C.ngrid[0], nb = C.ngrid[1], nc = C.ngrid[2];
  int al, ar, bl, br, cl, cr;
  double wal, war, wbl, wbr, wcl, wcr;
  equitable_axis(na, fa, &al, &ar, &wal, &war);
  equitable_axis(nb, fb, &bl, &br, &wbl, &wbr);
  equitable_axis(nc, fc, &cl, &cr, &wcl, &wcr);
  auto at = [&](int a, int b, int c) -> double& { return g[((size_t)a * nb + b) * nc + c]; };
  at(al, bl, cl) += wal * wbl * wcl;
  at(ar, bl, cl) += war * wbl * wcl;
  at(al, br, cl) += wal * wbr * wcl;
  at(al, bl, cr) += wal * wbl * wcr;
  at(ar, br, cl) += war * wbr * wcl;
  at(ar, bl, cr) += war * wbl * wcr;
  at(al, br, cr) += wal * wbr * wcr;
  at(ar, br, cr) += war * wbr * wcr;
}
static double frac_mod(double x) { return x - std::floor(x); }  // modulo(x, 1.0)
static void com(const MolType& M, int natms, const double* x, const double* y, const double* z, double* cx,
                double* cy, double* cz);
// storeprob (utility_pack.f:496-561): every guest molecule's centre of mass and sites in
// fractional coordinates, binned into the plots of its species.
static void storeprob(Chain& C) {
  double rcell[9], det;
  invert(C.cell, rcell, &det);
  for (int g = 0; g < C.ntpguest; g++) {
    const MolType& M = C.mols[C.locguest[g]];
    const int natms = M.numatoms;
    for (int m = 0; m < M.nummols; m++) {
      const double* x = M.fx.data() + m * natms;
      const double* y = M.fy.data() + m * natms;
      const double* z = M.fz.data() + m * natms;
      double cx, cy, cz;
      com(M, natms, x, y, z, &cx, &cy, &cz);
      double fc[3] = {frac_mod(cx * rcell[0] + cy * rcell[3] + cz * rcell[6]),
                      frac_mod(cx * rcell[1] + cy * rcell[4] + cz * rcell[7]),
                      frac_mod(cx * rcell[2] + cy * rcell[5] + cz * rcell[8])};
      for (size_t ip = 0; ip < C.plots.size(); ip++) {
        if (C.plots[ip].guest != g) continue;
        for (int site : C.plots[ip].sites) {
          if (site == 0) {
            equitable_bin(C, fc[0], fc[1], fc[2], C.grid[ip]);
          } else {
            const int j = site - 1;
            double fa = frac_mod(x[j] * rcell[0] + y[j] * rcell[3] + z[j] * rcell[6]);
            double fb = frac_mod(x[j] * rcell[1] + y[j] * rcell[4] + z[j] * rcell[7]);
            double fz = frac_mod(x[j] * rcell[2] + y[j] * rcell[5] + z[j] * rcell[8]);
            equitable_bin(C, fa, fb, fz, C.grid[ip]);
          }
        }
      }
    }
  }
}
// random_disp utility_pack.f:2679-2763 + random_rot 2929-3000
static void random_disp(Chain& C, const MolType& M, int natms, double delr, const double* rcell, double rotangle,
                        double ra, double rb, double rcc, double r1, double r2, double r3, double r4) {
  double half = delr * 0.5;
  ra = (2.0 * ra - 1.0) * half;
  rb = (2.0 * rb - 1.0) * half;
  rcc = (2.0 * rcc - 1.0) * half;
  double* x = C.newx.data();
  double* y = C.newy.data();
  double* z = C.newz.data();
  for (int i = 0; i < natms; i++) {
    x[i] = ra + x[i];
    y[i] = rb + y[i];
    z[i] = rcc + z[i];
  }
  double cx, cy, cz;
  com(M, natms, x, y, z, &cx, &cy, &cz);
  double ssx = (rcell[0] * cx + rcell[3] * cy + rcell[6] * cz);
  double ssy = (rcell[1] * cx + rcell[4] * cy + rcell[7] * cz);
  double ssz = (rcell[2] * cx + rcell[5] * cy + rcell[8] * cz);
  double xss = ssx - std::floor(ssx), yss = ssy - std::floor(ssy), zss = ssz - std::floor(ssz);
  const double* cell = C.cell;
  double wx = (cell[0] * xss + cell[3] * yss + cell[6] * zss);
  double wy = (cell[1] * xss + cell[4] * yss + cell[7] * zss);
  double wz = (cell[2] * xss + cell[5] * yss + cell[8] * zss);
  double sx = wx - cx, sy = wy - cy, sz = wz - cz;
  cx = wx;
  cy = wy;
  cz = wz;
  for (int i = 0; i < natms; i++) {
    x[i] = x[i] + sx;
    y[i] = y[i] + sy;
    z[i] = z[i] + sz;
  }
  // random_rot
  for (int i = 0; i < natms; i++) {
    x[i] = x[i] - cx;
    y[i] = y[i] - cy;
    z[i] = z[i] - cz;
  }
  double theta = r1 * rotangle, q[4];
  quat_from(theta, r2, r3, r4, q);
  rotation(x, y, z, natms, q[0], q[1], q[2], q[3]);
  for (int i = 0; i < natms; i++) {
    x[i] = x[i] + cx;
    y[i] = y[i] + cy;
    z[i] = z[i] + cz;
  }
}
// random_jump (utility_pack.f:2766-2813) + random_rot (2929-3000) with rotangle = 8 atan(1):
// the centre of mass moves to the cell point of fractional (ra, rb, rc), then the molecule
// turns about it.
static void random_jump(Chain& C, const MolType& M, int natms, double ra, double rb, double rcc, double r1,
                        double r2, double r3, double r4) {
  double* x = C.newx.data();
  double* y = C.newy.data();
  double* z = C.newz.data();
  const double* cell = C.cell;
  double xd = ra * cell[0] + rb * cell[3] + rcc * cell[6];
  double yd = ra * cell[1] + rb * cell[4] + rcc * cell[7];
  double zd = ra * cell[2] + rb * cell[5] + rcc * cell[8];
  double cx, cy, cz;
  com(M, natms, x, y, z, &cx, &cy, &cz);
  xd = xd - cx;
  yd = yd - cy;
  zd = zd - cz;
  for (int i = 0; i < natms; i++) {
    x[i] = xd + x[i];
    y[i] = yd + y[i];
    z[i] = zd + z[i];
  }
  com(M, natms, x, y, z, &cx, &cy, &cz);
  for (int i = 0; i < natms; i++) {
    x[i] = x[i] - cx;
    y[i] = y[i] - cy;
    z[i] = z[i] - cz;
  }
  const double jumpangle = 8.0 * std::atan(1.0);
  double theta = r1 * jumpangle, q[4];
  quat_from(theta, r2, r3, r4, q);
  rotation(x, y, z, natms, q[0], q[1], q[2], q[3]);
  for (int i = 0; i < natms; i++) {
    x[i] = x[i] + cx;
    y[i] = y[i] + cy;
    z[i] = z[i] + cz;
  }
}
// energy_eval utility_pack.f:3049-3095
static bool energy_eval(double eng, double rande, double volm, double press, int ngsts, double temp, double beta,
                        int move) {
  double test = 0.0;
  if (-1 * beta * eng > 700.0)
    test = std::exp(700.0);
  else if (move == MV_DISPLACE)
    test = std::exp(-1.0 * beta * eng);
  else if (move == MV_INSERT)
    test = volm * press / ((ngsts + 1) * BOLTZ * temp) * std::exp(-1.0 * beta * eng);
  else if (move == MV_DELETE) {
    if (std::fabs(press) < 1e-7)
      test = 1.0;
    else
      test = ngsts * BOLTZ * temp / (volm * press) * std::exp(-1.0 * beta * eng);
  }
  return rande < test;
}

// ---------------------------------------------------------------- set-up (gcmc.f:178-563)
static void setup(Chain& C, const std::string& dir, int si, int sj, int sk, int sl) {
  initscan(C, dir);
  C.mxebuf = (2 * C.kmax1 + 1) * (2 * C.kmax2 + 1) * (2 * C.kmax3 + 1) - 1;
  C.maxvdw = std::max(C.ntpvdw, (C.mxatyp * (C.mxatyp + 1)) / 2);
  // alloc_config_arrays utility_pack.f:725-726
  C.mxgrid = std::max(1000, (int)(C.rvdw / 0.01 + 0.5) + 4);
  C.mxegrd = C.mxgrid;
  C.ltpvdw.assign(C.maxvdw + 2, -1);
  C.lstvdw.assign(C.maxvdw + 2, 0);
  C.prmvdw.assign(C.maxvdw + 2, std::vector<double>(5, 0.0));
  C.vvv.assign(C.maxvdw + 2, std::vector<double>(C.mxgrid + 1, 0.0));
  C.steadd.assign(C.maxvdw + 2, 0.0);
  readfield(C, dir);
  C.delr.assign(C.ntpguest, C.initdelr);
  readconfig(C, dir);
  C.framatm = C.totatm;
  C.statvolm = C.volm * 1e-30;
  readcontrol(C, dir);
  // move-frequency normalisation gcmc.f:282-331
  for (int i = 0; i < C.ntpguest; i++) {
    double nrm = C.mcinsf[i] + C.mcdelf[i] + C.mcdisf[i] + C.mcjmpf[i] + C.mcflxf[i] + C.mcswpf[i] + C.mctraf[i] +
                 C.mcrotf[i] + C.mcmjpf[i];
    if (nrm == 0) {
      nrm = 1;
      C.mcinsf[i] = 1.0 / 3.0;
      C.mcdelf[i] = 1.0 / 3.0;
      C.mcdisf[i] = 1.0 / 3.0;
      C.mcjmpf[i] = C.mcflxf[i] = C.mcswpf[i] = C.mctraf[i] = C.mcrotf[i] = C.mcmjpf[i] = 0.0;
    }
    C.mcinsf[i] = C.mcinsf[i] / nrm;
    C.mcdelf[i] = C.mcinsf[i] + (C.mcdelf[i] / nrm);
    C.mcdisf[i] = C.mcdelf[i] + (C.mcdisf[i] / nrm);
    C.mcjmpf[i] = C.mcdisf[i] + (C.mcjmpf[i] / nrm);
    C.mcflxf[i] = C.mcjmpf[i] + (C.mcflxf[i] / nrm);
    C.mcswpf[i] = C.mcflxf[i] + (C.mcswpf[i] / nrm);
    C.mctraf[i] = C.mcswpf[i] + (C.mctraf[i] / nrm);
    C.mcrotf[i] = C.mctraf[i] + (C.mcrotf[i] / nrm);
    C.mcmjpf[i] = C.mcrotf[i] + (C.mcmjpf[i] / nrm);
  }
  C.rng.seed(si, sj, sk, sl);
  C.rng.next();  // gcmc.f:335-336: the second duni() call consumes one draw
  C.rotangle = PI / 3.0;
  guest_exclude(C);
  condense(C);
  C.beta = 1.0 / (KBOLTZ * C.temp);
  C.epsq = 1.0;
  C.ckcsum.assign(C.mxebuf + 1, 0.0);
  C.ckssum.assign(C.mxebuf + 1, 0.0);
  C.ckcsnew.assign(C.mxebuf + 1, 0.0);
  C.ckssnew.assign(C.mxebuf + 1, 0.0);
  erfcgen(C);
  single_point(C);
  ewald1(C, C.mxatm, nullptr);  // gcmc.f:522-524: S(k) over all atoms present at start
  // ewald3en gcmc.f:529-552
  C.ewald3en.assign(C.ntpguest, 0.0);
  for (int k = 0; k < C.ntpguest; k++) {
    const MolType& M = C.mols[C.locguest[k]];
    int natms = M.numatoms;
    double sum = 0.0;
    for (int i = 0; i < natms - 1; i++) {
      std::vector<double> xd, yd, zd;
      std::vector<int> jl;
      for (int j = i + 1; j < natms; j++) {
        jl.push_back(j);
        xd.push_back(C.guestx[k][i] - C.guestx[k][j]);
        yd.push_back(C.guesty[k][i] - C.guesty[k][j]);
        zd.push_back(C.guestz[k][i] - C.guestz[k][j]);
      }
      images(C.imcon, (int)xd.size(), C.cell, xd.data(), yd.data(), zd.data());
      sum += ewald3(C, M.chg[i], (int)xd.size(), xd.data(), yd.data(), zd.data(),
                    [&](int m) { return M.chg[jl[m]]; });
    }
    C.ewald3en[k] = sum;
  }
  C.energy.assign(C.ntpguest, C.spenergy);
  C.delE.assign(C.ntpguest, 0.0);
  C.elrc = 0.0;  // the main program's elrc starts at zero (gcmc.f:131-132)
  C.delrdisp = C.delr;
  C.tran_delr = C.delr;
  C.rota_rotangle = C.rotangle;
  C.accept_disp.assign(C.ntpguest, 0);
  C.disp_count.assign(C.ntpguest, 0);
  C.accept_tran.assign(C.ntpguest, 0);
  C.tran_count.assign(C.ntpguest, 0);
  C.chainstats.assign(1 + 14 * C.ntpguest, 0.0);
  C.avgwindow.assign(8 * C.ntpguest, 0.0);
  C.sumwindowav.assign(8 * C.ntpguest, 0.0);
  C.varwindow.assign(8 * C.ntpguest, 0.0);
  C.seltot.assign(C.ntpguest * C.ntpguest, 0.0);
  C.selwin.assign(C.ntpguest * C.ntpguest, 0.0);
  C.gasmol.assign((size_t)C.ntpguest * 500000 + 1, 0.0);
  C.gaseng.assign((size_t)C.ntpguest * 500000 + 1, 0.0);
  if (!C.plots.empty()) {  // gcmc.f:246-265
    for (int i = 0; i < 3; i++)
      C.ngrid[i] = C.gridfactor[i] * (int)std::ceil(C.celprp[i] / (C.griddim * C.gridfactor[i]));
    C.grid.assign(C.plots.size(), std::vector<double>((size_t)C.ngrid[0] * C.ngrid[1] * C.ngrid[2], 0.0));
  }
  C.production = (C.eqsteps == 0);
  C.lgchk = !C.lspe;  // gcmc.f:565-567: a single-point deck stops before the move loop
  int maxs = 64;
  C.ind.assign(maxs, -1);
  C.newx.assign(maxs, 0.0);
  C.newy.assign(maxs, 0.0);
  C.newz.assign(maxs, 0.0);
}

static int guest_offset(const Chain& C, int iguest) {
  int atmadd = 0;
  for (int n = 0; n < iguest; n++) {
    const MolType& M = C.mols[C.locguest[n]];
    atmadd += M.numatoms * M.nummols;
  }
  return atmadd;
}

// One iteration of the move loop gcmc.f:589-1380 (+ statistics 1814-1860, no file output).
static void gcmc_step(Chain& C, MoveRec* rec) {
  C.gcmccount++;
  // termination / production switching every 400 steps (gcmc.f:594-736; one rank)
  if (C.gcmccount % 400 == 0) {
    int totalguests = 0;
    for (int i = 0; i < C.ntpguest; i++) totalguests += C.mols[C.locguest[i]].nummols;
    if (C.production) {
      if (C.mcsteps < 0) {
        for (int t = 4; t > 0; t--) C.tick_tock[t] = C.tick_tock[t - 1];
        C.tick_tock[0] = true;
        if (C.prodcount < (long long)(-C.mcsteps) * (totalguests + 1)) C.tick_tock[0] = false;
        bool all = true;
        for (bool b : C.tick_tock) all = all && b;
        if (all) C.lgchk = false;
      } else if (C.prodcount >= C.mcsteps) {
        C.lgchk = false;
      }
    } else {
      if (C.despre > 0) {  // pressure equilibration (gcmc.f:637-696)
        for (int t = 4; t > 0; t--) C.tick_tock[t] = C.tick_tock[t - 1];
        C.tick_tock[0] = true;
        if (C.prodcount < (long long)(-C.eqsteps) * (totalguests + 1) / 4) C.tick_tock[0] = false;
        if (C.tick_tock[0]) {
          const int ng = C.ntpguest;
          double totpres = 0.0;
          for (int i = 0; i < ng; i++) totpres += C.gstpress[i];
          for (int i = 0; i < ng; i++) {
            const int is = 14 * i, mol = C.locguest[i];
            double temppres = (C.gstpress[mol] * (1 - C.packf) * C.volm / C.packf) / (C.temp * 13806874.7924278);
            C.dqp[mol] = C.adsguen[mol] - C.chainstats[is + 1] + (C.adspres[mol] - temppres);
            C.chainstats[is + 1] = 0;
          }
          auto sum_dqp = [&C]() {
            double t = 0.0;
            for (double v : C.dqp) t += v;
            return t;
          };
          for (int i = 0; i < ng - 1; i++) {
            const int mol = C.locguest[i];
            C.presrate = C.dqp[mol] - sum_dqp() * C.gstpress[mol] / totpres;
            C.gstpress[mol] = C.dqp[mol] * totpres / sum_dqp();
            if (C.gstpress[mol] < 0) C.gstpress[mol] = 0;
            C.presleft = C.presleft + C.gstpress[mol];
          }
          C.gstpress[C.locguest[ng - 1]] = totpres - C.presleft;
          if (C.gstpress[C.locguest[ng - 1]] < 0) C.gstpress[C.locguest[ng - 1]] = 0;
          double sp = 0.0;
          for (int i = 0; i < ng; i++) sp += C.gstpress[i];
          const double changerate = totpres / sp;
          for (int i = 0; i < ng; i++) C.gstpress[C.locguest[i]] = C.gstpress[C.locguest[i]] * changerate;
          C.presleft = 0.0;
          C.prodcount = 0;
          if (std::fabs(C.presrate) < C.despre || (long long)C.gcmccount > -50LL * C.eqsteps) {
            C.gcmccount = 0;
            C.despre = 0;
          }
        }
      }
      if (C.eqsteps > 0) {
        if (C.gcmccount >= C.eqsteps && C.despre == 0) C.production = true;
      } else if (C.eqsteps < 0) {
        for (int t = 4; t > 0; t--) C.tick_tock[t] = C.tick_tock[t - 1];
        C.tick_tock[0] = true;
        if ((long long)C.gcmccount < (long long)(-C.eqsteps) * (totalguests + 1)) C.tick_tock[0] = false;
        if (C.despre > 0) C.tick_tock[0] = false;
        bool all = true;
        for (bool b : C.tick_tock) all = all && b;
        if (all) {
          C.production = true;
          for (bool& b : C.tick_tock) b = false;
        }
      }
    }
  }
  int iguest = 0;
  if (C.ntpguest > 1) iguest = (int)std::floor(C.rng.next() * C.ntpguest);
  double randmov = C.rng.next();
  bool insert = false, del = false, displace = false, tran = false, rota = false, jump = false, noop = false,
       mjump = false;
  if (randmov < C.mcinsf[iguest])
    insert = true;
  else if (randmov < C.mcdelf[iguest])
    del = true;
  else if (randmov < C.mcdisf[iguest])
    displace = true;
  else if (randmov < C.mcjmpf[iguest])
    jump = true;
  else if (randmov < C.mcflxf[iguest] || randmov < C.mcswpf[iguest])
    noop = true;  // flex and swap are not implemented by the reference (gcmc.f:1789-1795)
  else if (randmov < C.mctraf[iguest]) {
    displace = true;
    tran = true;
  } else if (randmov < C.mcrotf[iguest]) {
    displace = true;
    rota = true;
  } else if (randmov < C.mcmjpf[iguest])
    mjump = true;
  else
    displace = true;
  MolType& M = C.mols[C.locguest[iguest]];
  int natms = M.numatoms, nmols = M.nummols;
  // guest geometries before the move (gcmc.f:785-792, hisarchive 2491-2517)
  if (C.nhis != 0 && C.gcmccount % std::abs(C.nhis) == 0 && !C.his_f.empty() && (C.nhis < 0 || C.prodcount > 0))
    for (int k = 0; k < C.ntpguest; k++) {
      const MolType& G = C.mols[C.locguest[k]];
      std::fprintf(C.his_f[k], "%6d\nstep %7d\n", G.nummols * G.numatoms, C.gcmccount);
      for (int i = 0, iatm = 0; i < G.nummols; i++)
        for (int j = 0; j < G.numatoms; j++, iatm++)
          std::fprintf(C.his_f[k], "  %c%16.6f%16.6f%16.6f\n", G.atmname[j].empty() ? ' ' : G.atmname[j][0],
                       G.fx[iatm], G.fy[iatm], G.fz[iatm]);
    }
  // step-size adaptation gcmc.f:794-834 (applied on every pass while the counters sit on a
  // multiple of 50/100, as the reference does)
  if (nmols >= 1 && C.disp_count[iguest] >= 1) {
    if (C.disp_count[iguest] % 100 == 0) {
      if ((C.accept_disp[iguest] / (double)C.disp_count[iguest]) > C.disp_ratio[iguest])
        C.delrdisp[iguest] = C.delrdisp[iguest] * 1.05;
      else if (C.delrdisp[iguest] > DELRMIN)
        C.delrdisp[iguest] = C.delrdisp[iguest] * 0.95;
    } else if (C.disp_count[iguest] % 50 == 0) {
      if ((C.accept_disp[iguest] / (double)C.disp_count[iguest]) > C.disp_ratio[iguest])
        C.rotangle = C.rotangle * 1.05;
      else if (C.rotangle > MINANGLE)
        C.rotangle = C.rotangle * 0.95;
    }
  }
  if (nmols >= 1 && C.tran_count[iguest] >= 1 && C.tran_count[iguest] % 100 == 0) {
    if ((C.accept_tran[iguest] / (double)C.tran_count[iguest]) > C.tran_ratio[iguest])
      C.tran_delr[iguest] = C.tran_delr[iguest] * 1.05;
    else if (C.tran_delr[iguest] > DELRMIN)
      C.tran_delr[iguest] = C.tran_delr[iguest] * 0.95;
  }
  if (nmols >= 1 && C.rota_count >= 1 && C.rota_count % 100 == 0) {
    if ((C.accept_rota / (double)C.rota_count) > C.rota_ratio)
      C.rota_rotangle = C.rota_rotangle * 1.05;
    else if (C.rota_rotangle > MINANGLE)
      C.rota_rotangle = C.rota_rotangle * 0.95;
  }
  if (nmols == 0 || (nmols == 1 && mjump)) {  // gcmc.f:837-847
    insert = true;
    del = displace = tran = rota = jump = noop = mjump = false;
  }
  MoveRec R;
  std::memset(&R, 0, sizeof(R));
  R.step = C.gcmccount;
  R.iguest = iguest;
  R.randchoice = 0;
  bool accepted = false;
  double ewld1eng = 0, ewld2sum = 0, ewld3sum = 0, vdwsum = 0, delrc = 0, estep = 0, rande = -1;
  std::vector<double> chg(natms);
  std::vector<int> styp(natms);
  C.delE[iguest] = 0.0;
  if (insert) {
    R.mtype = 1;
    C.ins_count++;
    if ((C.totatm - C.framatm) + natms >= C.maxguest) fail(75, "too many atoms in specified system");
    double ra = C.rng.next(), rb = C.rng.next(), rc_ = C.rng.next();
    double r1 = C.rng.next(), r2 = C.rng.next(), r3 = C.rng.next(), r4 = C.rng.next();
    random_ins(C, iguest, natms, ra, rb, rc_, r1, r2, r3, r4);
    for (int i = 0; i < natms; i++) C.ind[i] = -1;
    ewld1eng = ewald1_guest(C, iguest, natms, C.newx.data(), C.newy.data(), C.newz.data(), MV_INSERT, 1);
    for (int i = 0; i < natms; i++) {
      C.numtyp[M.ltpsit[i]]++;
      if (M.frz[i] != 0) C.numfrz[M.ltpsit[i]]++;
    }
    delrc = gstlrcorrect(C);
    delrc = delrc - C.elrc;
    for (int i = 0; i < natms; i++) {
      chg[i] = M.chg[i];
      styp[i] = M.ltpsit[i];
    }
    guest_realspace(C, natms, C.newx.data(), C.newy.data(), C.newz.data(), C.ind.data(), chg.data(), styp.data(),
                    &ewld2sum, &vdwsum);
    ewld3sum = C.ewald3en[iguest];
    double gpress = C.gstpress[iguest];
    int ngsts = M.nummols;
    estep = (ewld1eng + ewld2sum + ewld3sum + vdwsum + delrc) / C.engunit;
    rande = C.rng.next();
    accepted = energy_eval(estep, rande, C.statvolm, gpress, ngsts, C.temp, C.beta, MV_INSERT);
    if (accepted) {
      C.delE[iguest] = estep;
      C.accept_ins++;
      int mm = natms * M.nummols;
      M.fx.resize(std::max<size_t>(M.fx.size(), mm + natms));
      M.fy.resize(std::max<size_t>(M.fy.size(), mm + natms));
      M.fz.resize(std::max<size_t>(M.fz.size(), mm + natms));
      for (int i = 0; i < natms; i++) {
        M.fx[mm + i] = C.newx[i];
        M.fy[mm + i] = C.newy[i];
        M.fz[mm + i] = C.newz[i];
      }
      for (int i = 0; i < C.newld; i++) {
        C.ckcsum[i] = C.ckcsnew[i];
        C.ckssum[i] = C.ckssnew[i];
      }
      C.elrc = C.elrc + delrc;
      M.nummols++;
      C.totatm += natms;
      condense(C);
      C.energy[iguest] += C.delE[iguest];
    } else {
      for (int i = 0; i < natms; i++) {
        C.numtyp[M.ltpsit[i]]--;
        if (M.frz[i] != 0) C.numfrz[M.ltpsit[i]]--;
      }
    }
  } else if (del) {
    R.mtype = 2;
    C.del_count++;
    int randchoice = (int)std::floor(C.rng.next() * nmols) + 1;
    R.randchoice = randchoice;
    int atmadd = guest_offset(C, iguest);
    int at = (randchoice - 1) * natms;  // 0-based first atom of the molecule
    for (int k = 0; k < natms; k++) {
      C.ind[k] = atmadd + at + k;
      C.newx[k] = M.fx[at + k];
      C.newy[k] = M.fy[at + k];
      C.newz[k] = M.fz[at + k];
    }
    for (int i = 0; i < natms; i++) {
      C.numtyp[M.ltpsit[i]]--;
      if (M.frz[i] != 0) C.numfrz[M.ltpsit[i]]--;
    }
    delrc = gstlrcorrect(C);
    delrc = delrc - C.elrc;
    ewld1eng = ewald1_guest(C, iguest, natms, C.newx.data(), C.newy.data(), C.newz.data(), MV_DELETE, 1);
    for (int i = 0; i < natms; i++) {
      chg[i] = C.atmcharge[C.ind[i]];
      styp[i] = C.ltype[C.ind[i]];
    }
    guest_realspace(C, natms, C.newx.data(), C.newy.data(), C.newz.data(), C.ind.data(), chg.data(), styp.data(),
                    &ewld2sum, &vdwsum);
    ewld3sum = C.ewald3en[iguest];
    double gpress = C.gstpress[iguest];
    int ngsts = M.nummols;
    estep = (ewld1eng - ewld2sum - ewld3sum - vdwsum + delrc) / C.engunit;
    rande = C.rng.next();
    accepted = energy_eval(estep, rande, C.statvolm, gpress, ngsts, C.temp, C.beta, MV_DELETE);
    if (accepted) {
      C.delE[iguest] = estep;
      C.accept_del++;
      int mm = natms * M.nummols;
      for (int i = at + natms; i < mm; i++) {
        M.fx[i - natms] = M.fx[i];
        M.fy[i - natms] = M.fy[i];
        M.fz[i - natms] = M.fz[i];
      }
      for (int i = 0; i < C.newld; i++) {
        C.ckcsum[i] = C.ckcsnew[i];
        C.ckssum[i] = C.ckssnew[i];
      }
      C.elrc = C.elrc + delrc;
      M.nummols--;
      C.totatm -= natms;
      condense(C);
      C.energy[iguest] += C.delE[iguest];
    } else {
      for (int i = 0; i < natms; i++) {
        C.numtyp[M.ltpsit[i]]++;
        if (M.frz[i] != 0) C.numfrz[M.ltpsit[i]]++;
      }
    }
  } else if (displace) {
    double ra, rb, rc_, r1, r2, r3, r4, dis_delr, dis_rot;
    if (tran) {
      R.mtype = 4;
      C.tran_count[iguest]++;
      ra = C.rng.next();
      rb = C.rng.next();
      rc_ = C.rng.next();
      r1 = r2 = r3 = r4 = 0.0;
      dis_delr = C.tran_delr[iguest];
      dis_rot = 0.0;
    } else if (rota) {
      R.mtype = 5;
      C.rota_count++;
      ra = rb = rc_ = 0.5;
      r1 = C.rng.next();
      r2 = C.rng.next();
      r3 = C.rng.next();
      r4 = C.rng.next();
      dis_delr = 0.0;
      dis_rot = C.rota_rotangle;
    } else {
      R.mtype = 3;
      C.disp_count[iguest]++;
      ra = C.rng.next();
      rb = C.rng.next();
      rc_ = C.rng.next();
      r1 = C.rng.next();
      r2 = C.rng.next();
      r3 = C.rng.next();
      r4 = C.rng.next();
      dis_delr = C.delrdisp[iguest];
      dis_rot = C.rotangle;
    }
    int randchoice = (int)std::floor(C.rng.next() * nmols) + 1;
    R.randchoice = randchoice;
    int atmadd = guest_offset(C, iguest);
    int at = (randchoice - 1) * natms;
    for (int k = 0; k < natms; k++) {
      C.ind[k] = atmadd + at + k;
      C.newx[k] = M.fx[at + k];
      C.newy[k] = M.fy[at + k];
      C.newz[k] = M.fz[at + k];
    }
    ewald1_guest(C, iguest, natms, C.newx.data(), C.newy.data(), C.newz.data(), MV_DISPLACE, 1);
    for (int i = 0; i < natms; i++) {
      chg[i] = C.atmcharge[C.ind[i]];
      styp[i] = C.ltype[C.ind[i]];
    }
    // gcmc.f:1270-1278 subtracts site by site; the per-site sums are added in site order
    // inside guest_realspace, so replay that order here.
    {
      std::vector<double> se(natms), sv(natms);
      double a, b;
      guest_realspace(C, natms, C.newx.data(), C.newy.data(), C.newz.data(), C.ind.data(), chg.data(),
                      styp.data(), &a, &b, se.data(), sv.data());
      ewld2sum = 0.0;
      vdwsum = 0.0;
      for (int i = 0; i < natms; i++) {
        ewld2sum = ewld2sum - se[i];
        vdwsum = vdwsum - sv[i];
      }
    }
    double rcell[9], det;
    invert(C.cell, rcell, &det);
    random_disp(C, M, natms, dis_delr, rcell, dis_rot, ra, rb, rc_, r1, r2, r3, r4);
    ewld1eng = ewald1_guest(C, iguest, natms, C.newx.data(), C.newy.data(), C.newz.data(), MV_DISPLACE, 2);
    {
      std::vector<double> se(natms), sv(natms);
      double a, b;
      guest_realspace(C, natms, C.newx.data(), C.newy.data(), C.newz.data(), C.ind.data(), chg.data(),
                      styp.data(), &a, &b, se.data(), sv.data());
      for (int i = 0; i < natms; i++) {
        ewld2sum = ewld2sum + se[i];
        vdwsum = vdwsum + sv[i];
      }
    }
    estep = (ewld1eng + ewld2sum + vdwsum) / C.engunit;
    if (estep < 0.0) {
      accepted = true;
    } else {
      rande = C.rng.next();
      accepted = energy_eval(estep, rande, C.statvolm, C.gstpress[iguest], M.nummols, C.temp, C.beta, MV_DISPLACE);
    }
    if (accepted) {
      C.delE[iguest] = estep;
      if (tran)
        C.accept_tran[iguest]++;
      else if (rota)
        C.accept_rota++;
      else
        C.accept_disp[iguest]++;
      for (int j = 0; j < natms; j++) {
        M.fx[at + j] = C.newx[j];
        M.fy[at + j] = C.newy[j];
        M.fz[at + j] = C.newz[j];
      }
      for (int i = 0; i < C.newld; i++) {
        C.ckcsum[i] = C.ckcsnew[i];
        C.ckssum[i] = C.ckssnew[i];
      }
      condense(C);
      C.energy[iguest] += C.delE[iguest];
    }
  } else if (jump) {
    // long jump gcmc.f:1389-1547: the molecule leaves its place (pass 1) and reappears anywhere
    // in the cell with a random orientation (random_jump, pass 2)
    R.mtype = 6;
    C.jump_count++;
    int randchoice = (int)std::floor(C.rng.next() * nmols) + 1;
    R.randchoice = randchoice;
    int atmadd = guest_offset(C, iguest);
    int at = (randchoice - 1) * natms;
    for (int k = 0; k < natms; k++) {
      C.ind[k] = atmadd + at + k;
      C.newx[k] = M.fx[at + k];
      C.newy[k] = M.fy[at + k];
      C.newz[k] = M.fz[at + k];
    }
    ewald1_guest(C, iguest, natms, C.newx.data(), C.newy.data(), C.newz.data(), MV_DISPLACE, 1);
    for (int i = 0; i < natms; i++) {
      chg[i] = C.atmcharge[C.ind[i]];
      styp[i] = C.ltype[C.ind[i]];
    }
    {
      std::vector<double> se(natms), sv(natms);
      double a, b;
      guest_realspace(C, natms, C.newx.data(), C.newy.data(), C.newz.data(), C.ind.data(), chg.data(),
                      styp.data(), &a, &b, se.data(), sv.data());
      ewld2sum = 0.0;
      vdwsum = 0.0;
      for (int i = 0; i < natms; i++) {
        ewld2sum = ewld2sum - se[i];
        vdwsum = vdwsum - sv[i];
      }
    }
    double ra = C.rng.next(), rb = C.rng.next(), rc_ = C.rng.next();
    double r1 = C.rng.next(), r2 = C.rng.next(), r3 = C.rng.next(), r4 = C.rng.next();
    random_jump(C, M, natms, ra, rb, rc_, r1, r2, r3, r4);
    ewld1eng = ewald1_guest(C, iguest, natms, C.newx.data(), C.newy.data(), C.newz.data(), MV_DISPLACE, 2);
    {
      std::vector<double> se(natms), sv(natms);
      double a, b;
      guest_realspace(C, natms, C.newx.data(), C.newy.data(), C.newz.data(), C.ind.data(), chg.data(),
                      styp.data(), &a, &b, se.data(), sv.data());
      for (int i = 0; i < natms; i++) {
        ewld2sum = ewld2sum + se[i];
        vdwsum = vdwsum + sv[i];
      }
    }
    estep = (ewld1eng + ewld2sum + vdwsum) / C.engunit;
    if (estep < 0.0) {
      accepted = true;
    } else {
      rande = C.rng.next();
      accepted = energy_eval(estep, rande, C.statvolm, C.gstpress[iguest], M.nummols, C.temp, C.beta, MV_DISPLACE);
    }
    if (accepted) {
      C.delE[iguest] = estep;
      C.accept_jump++;
      for (int j = 0; j < natms; j++) {
        M.fx[at + j] = C.newx[j];
        M.fy[at + j] = C.newy[j];
        M.fz[at + j] = C.newz[j];
      }
      for (int i = 0; i < C.newld; i++) {
        C.ckcsum[i] = C.ckcsnew[i];
        C.ckssum[i] = C.ckssnew[i];
      }
      condense(C);
      C.energy[iguest] += C.delE[iguest];
    }
  } else if (mjump) {
    // multiple long jumps (gcmc.f:1557-1785): two distinct molecules jump one after the other,
    // the first one committed before the second is evaluated; one acceptance test on the summed
    // energy change, after which both stay or both return (framework and S(k) restored).
    R.mtype = 8;
    C.jump_count++;
    C.delE[iguest] = 0.0;
    estep = 0.0;
    const std::vector<double> ox = M.fx, oy = M.fy, oz = M.fz;
    const std::vector<double> ockc = C.ckcsum, ocks = C.ckssum;
    const double origenergy = C.energy[iguest];
    const int nummove = 2;
    std::vector<int> prev(nmols, 0);
    int at = 0;
    for (int mv = 1; mv <= nummove; mv++) {
      ewld1eng = ewld2sum = vdwsum = 0.0;
      int randchoice = 0;
      for (;;) {  // a molecule that has not jumped in this move
        randchoice = (int)std::floor(C.rng.next() * nmols) + 1;
        bool fresh = true;
        for (int p : prev) fresh = fresh && p != randchoice;
        if (fresh) {
          prev[mv - 1] = randchoice;
          break;
        }
      }
      R.randchoice = randchoice;
      int atmadd = guest_offset(C, iguest);
      at = (randchoice - 1) * natms;
      for (int k = 0; k < natms; k++) {
        C.ind[k] = atmadd + at + k;
        C.newx[k] = M.fx[at + k];
        C.newy[k] = M.fy[at + k];
        C.newz[k] = M.fz[at + k];
      }
      ewald1_guest(C, iguest, natms, C.newx.data(), C.newy.data(), C.newz.data(), MV_DISPLACE, 1);
      for (int i = 0; i < natms; i++) {
        chg[i] = C.atmcharge[C.ind[i]];
        styp[i] = C.ltype[C.ind[i]];
      }
      {
        std::vector<double> se(natms), sv(natms);
        double a, b;
        guest_realspace(C, natms, C.newx.data(), C.newy.data(), C.newz.data(), C.ind.data(), chg.data(),
                        styp.data(), &a, &b, se.data(), sv.data());
        for (int i = 0; i < natms; i++) {
          ewld2sum = ewld2sum - se[i];
          vdwsum = vdwsum - sv[i];
        }
      }
      double ra = C.rng.next(), rb = C.rng.next(), rc_ = C.rng.next();
      double r1 = C.rng.next(), r2 = C.rng.next(), r3 = C.rng.next(), r4 = C.rng.next();
      random_jump(C, M, natms, ra, rb, rc_, r1, r2, r3, r4);
      ewld1eng = ewald1_guest(C, iguest, natms, C.newx.data(), C.newy.data(), C.newz.data(), MV_DISPLACE, 2);
      {
        std::vector<double> se(natms), sv(natms);
        double a, b;
        guest_realspace(C, natms, C.newx.data(), C.newy.data(), C.newz.data(), C.ind.data(), chg.data(),
                        styp.data(), &a, &b, se.data(), sv.data());
        for (int i = 0; i < natms; i++) {
          ewld2sum = ewld2sum + se[i];
          vdwsum = vdwsum + sv[i];
        }
      }
      estep = estep + (ewld1eng + ewld2sum + vdwsum) / C.engunit;
      if (mv < nummove) {  // the state after this jump is the next jump's starting point
        C.delE[iguest] = estep;
        for (int j = 0; j < natms; j++) {
          M.fx[at + j] = C.newx[j];
          M.fy[at + j] = C.newy[j];
          M.fz[at + j] = C.newz[j];
        }
        for (int i = 0; i < C.newld; i++) {
          C.ckcsum[i] = C.ckcsnew[i];
          C.ckssum[i] = C.ckssnew[i];
        }
        condense(C);
        C.energy[iguest] = origenergy + C.delE[iguest];
      }
    }
    if (estep < 0.0) {
      accepted = true;
    } else {
      rande = C.rng.next();
      accepted = energy_eval(estep, rande, C.statvolm, C.gstpress[iguest], M.nummols, C.temp, C.beta, MV_DISPLACE);
    }
    if (accepted) {
      C.delE[iguest] = estep;
      C.accept_jump++;
      for (int j = 0; j < natms; j++) {
        M.fx[at + j] = C.newx[j];
        M.fy[at + j] = C.newy[j];
        M.fz[at + j] = C.newz[j];
      }
      for (int i = 0; i < C.newld; i++) {
        C.ckcsum[i] = C.ckcsnew[i];
        C.ckssum[i] = C.ckssnew[i];
      }
      condense(C);
      C.energy[iguest] = origenergy + C.delE[iguest];
    } else {
      C.delE[iguest] = 0.0;
      M.fx = ox;
      M.fy = oy;
      M.fz = oz;
      C.ckcsum = ockc;
      C.ckssum = ocks;
      condense(C);
      C.energy[iguest] = origenergy;
    }
  } else if (noop) {
    R.mtype = 7;
    accepted = C.last_accepted;  // the reference leaves `accepted` as the last move set it
  }
  C.last_accepted = accepted;
  // running loading while the pressures equilibrate (gcmc.f:1796-1808)
  if (!C.production && C.despre > 0 && ((C.laccsample && accepted) || !C.laccsample)) {
    C.prodcount++;
    for (int i = 0; i < C.ntpguest; i++) {
      const double dm = (double)(float)C.mols[C.locguest[i]].nummols;
      double* a = &C.chainstats[14 * i + 1];
      *a = *a + (dm - *a) / (double)C.prodcount;
    }
  }
  // production statistics gcmc.f:1814-1860 (rolling <N>,<E>,<EN>,<N^2>,<E^2>)
  if (C.production) {
    if ((C.laccsample && accepted) || !C.laccsample) {
      C.prodcount++;
      C.rollcount++;
      C.chainstats[0] = (double)C.prodcount;
      for (int i = 0; i < C.ntpguest; i++) {
        double dm = (double)(float)C.mols[C.locguest[i]].nummols;
        double m2 = dm * dm, e = C.energy[i], e2 = e * e;
        if (C.prodcount <= 500001) {
          C.gasmol[(size_t)i * 500000 + C.prodcount - 1] = dm;
          C.gaseng[(size_t)i * 500000 + C.prodcount - 1] = e;
        }
        int is = 14 * i;
        double* cs = C.chainstats.data();
        double pc = (double)C.prodcount;
        double delta = dm - cs[is + 1];
        cs[is + 1] = cs[is + 1] + delta / pc;
        delta = e - cs[is + 2];
        cs[is + 2] = cs[is + 2] + delta / pc;
        delta = e * dm - cs[is + 3];
        cs[is + 3] = cs[is + 3] + delta / pc;
        delta = m2 - cs[is + 4];
        cs[is + 4] = cs[is + 4] + delta / pc;
        delta = e2 - cs[is + 5];
        cs[is + 5] = cs[is + 5] + delta / pc;
        double* aw = C.avgwindow.data() + 8 * i;
        if (insert && iguest == i && accepted) {  // rolling <exp(-dE/kT)> (gcmc.f:1856-1866)
          double h = std::exp(-1.0 * C.delE[i] / KBOLTZ / C.temp);
          C.ins_rollcount++;
          delta = h - cs[is + 6];
          h = cs[is + 6] + delta / C.accept_ins;
          cs[is + 6] = h;
          aw[7] = ((C.ins_rollcount - 1) * aw[7] + h) / (double)C.ins_rollcount;
        }
        const double rc = (double)C.rollcount;
        aw[0] = ((C.rollcount - 1) * aw[0] + dm) / rc;
        aw[1] = ((C.rollcount - 1) * aw[1] + e) / rc;
        aw[2] = ((C.rollcount - 1) * aw[2] + e * dm) / rc;
        aw[3] = ((C.rollcount - 1) * aw[3] + m2) / rc;
        aw[4] = ((C.rollcount - 1) * aw[4] + e2) / rc;
      }
    }
    if (C.prodcount % C.nwind == 0 || !C.lgchk) {  // close a window (gcmc.f:1887-1928)
      C.avcount++;
      const double weight = (double)C.rollcount / (double)C.nwind;
      const int ng = C.ntpguest;
      for (int i = 0; i < ng; i++) {
        const double* cs = C.chainstats.data() + 14 * i;
        double* aw = C.avgwindow.data() + 8 * i;
        aw[5] = calc_qst(cs[5], cs[2], cs[1], cs[4], cs[3], C.temp);
        aw[6] = calc_cv(cs[5], cs[2], cs[1], cs[4], cs[3], C.temp);
        if (i > 0) {
          const double an = aw[0];
          for (int j = 0; j < i; j++) {
            if (an == 0) continue;
            double sel = C.avgwindow[8 * j] / an;
            double& st = C.seltot[i * ng + j];
            double& sw = C.selwin[i * ng + j];
            double delta = weight * (sel - st);
            st = st + delta / C.avcount;
            sw = sw + weight * (sel * sel - sw) / (C.avcount - 1 + weight);
            C.seltot[j * ng + i] = ((C.avcount - 1 + weight) * sw - ((C.avcount - 1 + weight) * st * st)) /
                                   (C.avcount - 1 + weight);
          }
        }
      }
      for (int k = 0; k < 8 * ng; k++) {
        double delta = weight * (C.avgwindow[k] - C.sumwindowav[k]);
        C.sumwindowav[k] = C.sumwindowav[k] + delta / C.avcount;
        C.varwindow[k] = C.varwindow[k] + delta * weight * (C.avgwindow[k] - C.sumwindowav[k]);
        C.avgwindow[k] = 0.0;
      }
      C.rollcount = 0;
    }
    if (!C.plots.empty()) storeprob(C);  // gcmc.f:1929-1931, every production move
  }
  // numguests.out (gcmc.f:1937-1951): only the moved species carries its dE and move flags,
  // the others' were cleared when their last move ended
  if (!C.numg_f.empty() && C.gcmccount % C.nnumg == 0) {
    const int fl[6] = {insert ? 1 : 0, del ? 1 : 0, displace ? (tran ? 2 : rota ? 3 : 1) : 0,
                       jump ? 1 : mjump ? 2 : 0, 0, 0};
    for (int i = 0; i < C.ntpguest; i++) {
      const bool me = i == iguest;
      std::fprintf(C.numg_f[i], "%9d%7d%20.6f%20.6f%4d%4d%4d%4d%4d%4d\n", C.gcmccount,
                   C.mols[C.locguest[i]].nummols, C.energy[i], me ? C.delE[i] : 0.0, me ? fl[0] : 0,
                   me ? fl[1] : 0, me ? fl[2] : 0, me ? fl[3] : 0, me ? fl[4] : 0, me ? fl[5] : 0);
    }
  }
  R.accepted = accepted ? 1 : 0;
  R.nmols_after = M.nummols;
  R.ewld1 = ewld1eng;
  R.ewld2 = ewld2sum;
  R.ewld3 = ewld3sum;
  R.vdw = vdwsum;
  R.delrc = delrc;
  R.estep = estep;
  R.rande = rande;
  R.energy_after = C.energy[iguest];
  if (rec) *rec = R;
}

}  // namespace orc

// ================================================================= C ABI for the tests
using namespace orc;

struct OrcHandle {
  Chain C;
  std::string err;
  void close_outputs() {
    for (FILE* f : C.numg_f)
      if (f) std::fclose(f);
    for (FILE* f : C.his_f)
      if (f) std::fclose(f);
    C.numg_f.clear();
    C.his_f.clear();
  }
  ~OrcHandle() { close_outputs(); }
};

static thread_local std::string g_last_error;

extern "C" {

const char* orc_last_error() { return g_last_error.c_str(); }

// Opens a CONTROL/FIELD/CONFIG directory, runs the reference's set-up up to the first move,
// and seeds duni with (i,j,k,l).  Returns nullptr on error (orc_last_error(), *code).
void* orc_open(const char* dir, int si, int sj, int sk, int sl, int* code) {
  OrcHandle* h = new OrcHandle();
  try {
    setup(h->C, dir, si, sj, sk, sl);
    if (code) *code = 0;
    return h;
  } catch (const FmcError& e) {
    g_last_error = e.msg;
    if (code) *code = e.code;
  } catch (const std::exception& e) {
    g_last_error = e.what();
    if (code) *code = -1;
  }
  delete h;
  return nullptr;
}

void orc_close(void* p) { delete (OrcHandle*)p; }
// Opens numguests.out and, when the deck asks for a history, his.xyz in `dir` (numguestsNN.out
// and hisNN.xyz per species for mixtures, gcmc.f:418-450); a null dir closes them.
int orc_open_outputs(void* p, const char* dir) {
  OrcHandle* h = (OrcHandle*)p;
  Chain& C = h->C;
  h->close_outputs();
  if (!dir) return 0;
  const int ng = C.ntpguest;
  for (int i = 0; i < ng; i++) {
    char a[64], b[64];
    if (ng > 1) {
      std::snprintf(a, sizeof(a), "/numguests%02d.out", i + 1);
      std::snprintf(b, sizeof(b), "/his%02d.xyz", i + 1);
    } else {
      std::snprintf(a, sizeof(a), "/numguests.out");
      std::snprintf(b, sizeof(b), "/his.xyz");
    }
    C.numg_f.push_back(std::fopen((std::string(dir) + a).c_str(), "w"));
    if (C.nhis != 0) C.his_f.push_back(std::fopen((std::string(dir) + b).c_str(), "w"));
  }
  for (FILE* f : C.numg_f)
    if (!f) return -1;
  for (FILE* f : C.his_f)
    if (!f) return -1;
  return 0;
}

// Scalars: [0] alpha [1] rcut [2] delr [3] volm [4] engunit [5] temp [6] beta [7] drewd
// [8] dlrpot [9] spenergy [10] dlpeng [11] ewald1sum [12] elrc [13] energy(1) [14] statvolm
void orc_scalars(void* p, double* out) {
  Chain& C = ((OrcHandle*)p)->C;
  double v[15] = {C.alpha, C.rcut, C.delr.empty() ? 0 : C.delr[0], C.volm, C.engunit, C.temp, C.beta, C.drewd,
                  C.dlrpot, C.spenergy, C.dlpeng, C.ewald1sum, C.elrc, C.energy.empty() ? 0 : C.energy[0],
                  C.statvolm};
  std::memcpy(out, v, sizeof(v));
}
// Partial pressures (Pa) per guest, then the remaining pressure-equilibration tolerance.
void orc_pressures(void* p, double* out) {
  Chain& C = ((OrcHandle*)p)->C;
  for (int i = 0; i < C.ntpguest; i++) out[i] = C.gstpress[i];
  out[C.ntpguest] = C.despre;
}
// Integers: [0] imcon [1] kmax1 [2] kmax2 [3] kmax3 [4] newld [5] totatm [6] ntpguest
// [7] ntpatm [8] mxgrid [9] framatm-equivalent (framework atoms) [10] gcmccount [11] maxvdw
void orc_ints(void* p, int* out) {
  Chain& C = ((OrcHandle*)p)->C;
  int nf = 0;
  for (int t = 0; t < C.ntpfram; t++) nf += C.mols[C.locfram[t]].nummols * C.mols[C.locfram[t]].numatoms;
  int v[12] = {C.imcon, C.kmax1, C.kmax2, C.kmax3, C.newld, C.totatm, C.ntpguest, C.ntpatm, C.mxgrid, nf,
               C.gcmccount, C.maxvdw};
  std::memcpy(out, v, sizeof(v));
}
// k-vector table in the reference's enumeration order: lmn[3K], akk[K]
int orc_kvectors(void* p, int* lmn, double* akk) {
  Chain& C = ((OrcHandle*)p)->C;
  double ralph = -0.25 / (C.alpha * C.alpha);
  bool lconsw = lconsw_of(C.imcon);
  double zero = 0.0;
  int K = 0;
  recip_walk(C, &zero, &zero, &zero, &zero, 1, [&](int kkk, int l, int m, int n, double rksq, double, double) {
    if (lmn) {
      lmn[3 * kkk] = l;
      lmn[3 * kkk + 1] = m;
      lmn[3 * kkk + 2] = n;
    }
    double rrksq = 1.0 / rksq;
    if (akk) akk[kkk] = lconsw ? std::exp(ralph * rksq) * rrksq : 4.0 * std::exp(ralph * rksq) * rrksq;
    K = kkk + 1;
  });
  return K;
}
int orc_sk(void* p, double* re, double* im) {
  Chain& C = ((OrcHandle*)p)->C;
  for (int i = 0; i < C.newld; i++) {
    re[i] = C.ckcsum[i];
    im[i] = C.ckssum[i];
  }
  return C.newld;
}
int orc_sknew(void* p, double* re, double* im) {
  Chain& C = ((OrcHandle*)p)->C;
  for (int i = 0; i < C.newld; i++) {
    re[i] = C.ckcsnew[i];
    im[i] = C.ckssnew[i];
  }
  return C.newld;
}
// Condensed atoms: xyz[3N] (interleaved), q[N], type[N] (1-based), frozen[N]
int orc_atoms(void* p, double* xyz, double* q, int* typ, int* frz) {
  Chain& C = ((OrcHandle*)p)->C;
  for (int i = 0; i < C.totatm; i++) {
    if (xyz) {
      xyz[3 * i] = C.xxx[i];
      xyz[3 * i + 1] = C.yyy[i];
      xyz[3 * i + 2] = C.zzz[i];
    }
    if (q) q[i] = C.atmcharge[i];
    if (typ) typ[i] = C.ltype[i];
    if (frz) frz[i] = C.lfreezesite[i];
  }
  return C.totatm;
}
// Tables: erc[0..mxegrd], vvv of one table id [0..mxgrid], pair map lstvdw[1..ntab]
int orc_erc(void* p, double* out) {
  Chain& C = ((OrcHandle*)p)->C;
  for (int i = 0; i <= C.mxegrd; i++) out[i] = C.erc[i];
  return C.mxegrd + 1;
}
int orc_vvv(void* p, int k, double* out) {
  Chain& C = ((OrcHandle*)p)->C;
  for (int i = 0; i <= C.mxgrid; i++) out[i] = C.vvv[k][i];
  return C.mxgrid + 1;
}
int orc_lstvdw(void* p, int* out) {
  Chain& C = ((OrcHandle*)p)->C;
  int ntab = C.ntpatm * (C.ntpatm + 1) / 2;
  for (int i = 1; i <= ntab; i++) out[i - 1] = C.lstvdw[i];
  return ntab;
}
// Guest template of guest type g (after the COM shift): xyz[3n], q[n], type[n], mass[n]
int orc_guest_template(void* p, int g, double* xyz, double* q, int* typ, double* mass) {
  Chain& C = ((OrcHandle*)p)->C;
  const MolType& M = C.mols[C.locguest[g]];
  for (int i = 0; i < M.numatoms; i++) {
    xyz[3 * i] = C.guestx[g][i];
    xyz[3 * i + 1] = C.guesty[g][i];
    xyz[3 * i + 2] = C.guestz[g][i];
    q[i] = M.chg[i];
    typ[i] = M.ltpsit[i];
    mass[i] = M.wght[i];
  }
  return M.numatoms;
}
double orc_ewald3en(void* p, int g) { return ((OrcHandle*)p)->C.ewald3en[g]; }

// ewald1_guest for the given site coordinates (interleaved xyz) against the current S(k);
// fills S_new via the chain's ckcsnew/ckssnew (read with orc_sknew).
double orc_ewald1_guest(void* p, int iguest, int natms, const double* xyz, int move, int pass) {
  Chain& C = ((OrcHandle*)p)->C;
  std::vector<double> x(natms), y(natms), z(natms);
  for (int i = 0; i < natms; i++) {
    x[i] = xyz[3 * i];
    y[i] = xyz[3 * i + 1];
    z[i] = xyz[3 * i + 2];
  }
  return ewald1_guest(C, iguest, natms, x.data(), y.data(), z.data(), move, pass);
}
// Real space of sites (xyz) with charges/types of guest type g against all condensed atoms
// except the 0-based indices in ind[natms] (-1 = none).  Per-site values optional.
void orc_realspace(void* p, int g, int natms, const double* xyz, const int* ind, double* ewld2, double* vdw,
                   double* site_e2, double* site_vdw) {
  Chain& C = ((OrcHandle*)p)->C;
  const MolType& M = C.mols[C.locguest[g]];
  std::vector<double> x(natms), y(natms), z(natms), chg(natms);
  std::vector<int> st(natms);
  for (int i = 0; i < natms; i++) {
    x[i] = xyz[3 * i];
    y[i] = xyz[3 * i + 1];
    z[i] = xyz[3 * i + 2];
    chg[i] = M.chg[i];
    st[i] = M.ltpsit[i];
  }
  guest_realspace(C, natms, x.data(), y.data(), z.data(), ind, chg.data(), st.data(), ewld2, vdw, site_e2,
                  site_vdw);
}
// Runs n moves; trace (optional) receives one record per move.  Returns moves run, or -code.
int orc_run(void* p, int n, MoveRec* trace) {
  OrcHandle* h = (OrcHandle*)p;
  try {
    for (int i = 0; i < n; i++) gcmc_step(h->C, trace ? trace + i : nullptr);
    return n;
  } catch (const FmcError& e) {
    g_last_error = e.msg;
    return e.code > 0 ? -e.code : -9999;
  }
}
// Runs until the reference's termination rule (steps or cycles) fires or max_moves is hit.
long long orc_run_to_completion(void* p, long long max_moves) {
  OrcHandle* h = (OrcHandle*)p;
  long long n = 0;
  while (h->C.lgchk && n < max_moves) {
    gcmc_step(h->C, nullptr);
    n++;
  }
  return n;
}
int orc_sizeof_moverec() { return (int)sizeof(MoveRec); }
double orc_duni(void* p) { return ((OrcHandle*)p)->C.rng.next(); }
// Standalone duni stream for a seed (first real draw included, none discarded).
void orc_duni_stream(int si, int sj, int sk, int sl, int n, double* out) {
  Duni d;
  d.seed(si, sj, sk, sl);
  for (int i = 0; i < n; i++) out[i] = d.next();
}
// Guest coordinates of guest type g in the reference's framwk order: xyz[3*nmol*natms]
int orc_guest_coords(void* p, int g, double* xyz) {
  Chain& C = ((OrcHandle*)p)->C;
  const MolType& M = C.mols[C.locguest[g]];
  int n = M.nummols * M.numatoms;
  if (xyz)
    for (int i = 0; i < n; i++) {
      xyz[3 * i] = M.fx[i];
      xyz[3 * i + 1] = M.fy[i];
      xyz[3 * i + 2] = M.fz[i];
    }
  return M.nummols;
}
// Overwrites the guests of type g with nmol molecules (xyz interleaved) and recomputes the
// state the reference would have after reading them from CONFIG/REVIVE: condense, single
// point energy, S(k).  Used for the REVIVE known-answer test.
int orc_load_guests(void* p, int g, int nmol, const double* xyz) {
  Chain& C = ((OrcHandle*)p)->C;
  MolType& M = C.mols[C.locguest[g]];
  int n = nmol * M.numatoms;
  C.totatm += (nmol - M.nummols) * M.numatoms;
  M.nummols = nmol;
  M.fx.assign(std::max(n, 1), 0.0);
  M.fy.assign(std::max(n, 1), 0.0);
  M.fz.assign(std::max(n, 1), 0.0);
  for (int i = 0; i < n; i++) {
    M.fx[i] = xyz[3 * i];
    M.fy[i] = xyz[3 * i + 1];
    M.fz[i] = xyz[3 * i + 2];
  }
  condense(C);
  single_point(C);
  ewald1(C, C.totatm, nullptr);
  C.energy.assign(C.ntpguest, C.spenergy);
  return C.totatm;
}
// State a restart takes from REVIVE besides the coordinates (gcmc.f:353-418 with revread,
// utility_pack.f:1840-1878): the production flag, kept only when no positive equilibration
// count follows (gcmc.f:396-409) and forced when there is none at all (gcmc.f:553-554), and
// the chain statistics; prodcount starts again at zero (gcmc.f:143).
void orc_restart_flags(void* p, int production, const double* chainstats) {
  Chain& C = ((OrcHandle*)p)->C;
  C.production = production != 0;
  if (C.production && C.eqsteps > 0) C.production = false;
  if (C.eqsteps == 0) C.production = true;
  for (size_t i = 0; i < C.chainstats.size(); i++) C.chainstats[i] = chainstats[i];
  C.prodcount = 0;
}
// Final statistics of the report (gcmc.f:1960-2037) on a copy of the chain's statistics:
// out[1 + 14 g + 0..13] = <N>, <E>, <EN>, <N^2>, <E^2>, 6th slot, then the errors of N, E, EN,
// N^2, E^2, Q_st, Cv and the 6th slot; out[0] = production moves.  Up to 500,000 production
// moves the averages and errors come from 5 blocks of the stored samples (each block sums
// the nwind + 1 samples of an inclusive slice and divides by nwind, as the reference does);
// beyond, from the windows closed during the run.
void orc_final_stats(void* p, double* out) {
  Chain& C = ((OrcHandle*)p)->C;
  const int ng = C.ntpguest, windn = 5;
  std::vector<double> cs = C.chainstats, var = C.varwindow, sum = C.sumwindowav, avg = C.avgwindow;
  int avcount = C.avcount;
  if (C.prodcount > 0) {
    const double weight = cs[0];
    for (int i = 0; i < ng; i++) {
      const int is = 14 * i, vs = 8 * i;
      if (weight <= 500000) {
        const long long nw = (long long)weight / windn;
        avcount = windn;
        std::fill(var.begin(), var.end(), 0.0);
        std::fill(sum.begin(), sum.end(), 0.0);
        std::fill(avg.begin(), avg.end(), 0.0);
        for (int x = 1; x <= windn; x++) {
          const size_t y = (size_t)i * 500000 + (size_t)(x - 1) * nw;
          double an = 0, e = 0, en = 0, n2 = 0, e2 = 0;
          for (size_t k = y; k <= y + nw; k++) {
            double m = k < C.gasmol.size() ? C.gasmol[k] : 0.0, g = k < C.gaseng.size() ? C.gaseng[k] : 0.0;
            an += m;
            e += g;
            en += m * g;
            n2 += m * m;
            e2 += g * g;
          }
          avg[0] = an / nw;
          avg[1] = e / nw;
          avg[2] = en / nw;
          avg[3] = n2 / nw;
          avg[4] = e2 / nw;
          avg[5] = calc_qst(avg[4], avg[1], avg[0], avg[3], avg[2], C.temp);
          avg[6] = calc_cv(avg[4], avg[1], avg[0], avg[3], avg[2], C.temp);
          for (int z = 0; z < 7; z++) {
            double delta = avg[z] - sum[z];
            sum[z] = sum[z] + delta / x;
            var[vs + z] = var[vs + z] + delta * (avg[z] - sum[z]);
            avg[z] = 0.0;
          }
        }
        for (int z = 0; z < 6; z++) cs[is + 1 + z] = sum[z];
      }
      for (int z = 0; z < 8; z++) cs[is + 7 + z] = std::sqrt(var[vs + z] / avcount);
    }
  }
  std::memcpy(out, cs.data(), sizeof(double) * cs.size());
}
// Window state: avcount, rollcount, then sumwindowav[8 ng], varwindow[8 ng], avgwindow[8 ng]
// and seltot[ng ng].
void orc_window_stats(void* p, double* out) {
  Chain& C = ((OrcHandle*)p)->C;
  const int ng = C.ntpguest;
  out[0] = C.avcount;
  out[1] = C.rollcount;
  double* o = out + 2;
  for (int k = 0; k < 8 * ng; k++) {
    o[k] = C.sumwindowav[k];
    o[8 * ng + k] = C.varwindow[k];
    o[16 * ng + k] = C.avgwindow[k];
  }
  for (int k = 0; k < ng * ng; k++) o[24 * ng + k] = C.seltot[k];
}
// Probability plots: dims[0..3] = plots, na, nb, nc; grid of plot ip when out is non-null.
int orc_prob(void* p, int ip, int* dims, double* out) {
  Chain& C = ((OrcHandle*)p)->C;
  if (dims) {
    dims[0] = (int)C.plots.size();
    dims[1] = C.ngrid[0];
    dims[2] = C.ngrid[1];
    dims[3] = C.ngrid[2];
  }
  if (out && ip >= 0 && ip < (int)C.grid.size()) std::memcpy(out, C.grid[ip].data(), sizeof(double) * C.grid[ip].size());
  return 0;
}
// Rolling statistics of guest type g: <N>,<E>,<EN>,<N^2>,<E^2>, prodcount
void orc_stats(void* p, int g, double* out) {
  Chain& C = ((OrcHandle*)p)->C;
  for (int i = 0; i < 5; i++) out[i] = C.chainstats[14 * g + 1 + i];
  out[5] = (double)C.prodcount;
}
}
