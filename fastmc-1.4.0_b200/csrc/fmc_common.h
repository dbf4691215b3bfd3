// Host/device shared pieces of the GCMC trial-move path: constants, the duni generator,
// minimum-image conventions, trial-move generators and the acceptance test.  Everything here
// is plain arithmetic usable from the host move loop (plain path) and from the persistent
// batched kernel, so both make the same decisions from the same random numbers.
#pragma once
#include <cmath>
#include <cstdint>

#if defined(__CUDACC__)
#define FMC_HD __host__ __device__ __forceinline__
#else
#define FMC_HD inline
#endif

namespace fmc {

// Physical constants and limits, utility_pack.f:71-113
constexpr double kPi = 3.141592653589793;
constexpr double kSqrPi = 1.7724538509055159;
constexpr double kR4pie0 = 138935.4835;      // e^2/(4 pi eps0 A) in 10 J/mol
constexpr double kKboltz = 1.9872041e-3;     // kcal/mol/K
constexpr double kBoltz = 1.3806503e-23;     // J/K
constexpr double kMinAngle = kPi / 18.0;     // utility_pack.f:86
constexpr double kDelrMin = 0.1;             // utility_pack.f:90
constexpr int kMaxGuestSites = 50;           // mxguestsite, utility_pack.f:76
constexpr int kMaxGuestTypes = 4;

// kJump: long jump (gcmc.f:1389-1547); kNoop: flex and swap, which the reference selects but
// does not implement (gcmc.f:1789-1795); kMultiJump: two long jumps under one acceptance test
// (gcmc.f:1557-1785)
enum MoveType : int {
  kInsert = 1,
  kDelete = 2,
  kDisplace = 3,
  kTranslate = 4,
  kRotate = 5,
  kJump = 6,
  kNoop = 7,
  kMultiJump = 8
};

// ------------------------------------------------------------------ duni
// Marsaglia-Zaman-Tsang universal generator in IEEE single precision, as duni in
// gcmc.f:2712-2805, with the clock-derived seed replaced by an explicit (i,j,k,l).
struct Duni {
  float u[97];
  float c;
  int ir, jr;
};

FMC_HD void duni_seed(Duni& d, int i, int j, int k, int l) {
  d.ir = 97;
  d.jr = 33;
  for (int ii = 0; ii < 97; ii++) {
    float s = 0.0f, t = 0.5f;
    for (int jj = 0; jj < 24; jj++) {
      int m = (((i * j) % 179) * k) % 179;
      i = j;
      j = k;
      k = m;
      l = (53 * l + 1) % 169;
      if ((l * m) % 64 >= 32) s = s + t;
      t = 0.5f * t;
    }
    d.u[ii] = s;
  }
  d.c = 362436.0f / 16777216.0f;
}

FMC_HD double duni_next(Duni& d) {
  const float cd = 7654321.0f / 16777216.0f, cm = 16777213.0f / 16777216.0f;
  float uni = d.u[d.ir - 1] - d.u[d.jr - 1];
  if (uni < 0.0f) uni = uni + 1.0f;
  d.u[d.ir - 1] = uni;
  d.ir = d.ir - 1;
  if (d.ir == 0) d.ir = 97;
  d.jr = d.jr - 1;
  if (d.jr == 0) d.jr = 97;
  d.c = d.c - cd;
  if (d.c < 0.0f) d.c = d.c + cm;
  uni = uni - d.c;
  if (uni < 0.0f) uni = uni + 1.0f;
  return (double)uni;
}

// ------------------------------------------------------------------ cell geometry
struct CellGeom {
  double h[9];    // cell vectors a,b,c (cell(1..9) of the reference, a = h[0..2])
  double rh[9];   // inverse (invert, utility_pack.f:1417)
  double inv[3];  // 1/h[0], 1/h[4], 1/h[8]: the reciprocals images() forms once per call
  double hex[3];  // hexagonal prism (imcon 7): a/(2 rt3), a/rt3, rt3/a as images() forms them
  double slab[4];  // slab (imcon 6): the in-plane inverse r1, r2, r4, r5 as images() forms it
  // slab voxel layers along z: the lowest layer's bottom, the layer height and its inverse
  double zlo, dz, rdz;
  double volm;    // volume used by Ewald and acceptance
  int imcon;
};

// The reference's own truncated constants of images (utility_pack.f:1149-1150).
constexpr double kImgRt2 = 1.41421356623, kImgRt3 = 1.7320508075;

inline void cell_reciprocals(CellGeom& c) {
  c.inv[0] = 1.0 / c.h[0];
  c.inv[1] = 1.0 / c.h[4];
  c.inv[2] = 1.0 / c.h[8];
  c.hex[0] = c.h[0] / (kImgRt3 * 2.0);
  c.hex[1] = c.h[0] / kImgRt3;
  c.hex[2] = kImgRt3 / c.h[0];
  double det = c.h[0] * c.h[4] - c.h[1] * c.h[3];
  det = 1.0 / det;
  c.slab[0] = det * c.h[4];
  c.slab[1] = -det * c.h[1];
  c.slab[2] = -det * c.h[3];
  c.slab[3] = det * c.h[0];
}

// Fortran nint: nearest integer, halves away from zero.
FMC_HD double fnint(double x) { return round(x); }

// Minimum image of one separation vector (images, utility_pack.f:1138-1349) for imcon 1, 2, 3,
// the half-shift cells 4 (truncated octahedron), 5 (rhombic dodecahedron) and 7 (hexagonal
// prism) and the slab 6, for a boundary condition known at compile time (other values: no
// image).
template <int kImcon>
FMC_HD void min_image_t(const CellGeom& c, double& x, double& y, double& z) {
  if (kImcon == 1) {
    const double a = c.h[0], ra = c.inv[0];
    x = x - a * fnint(ra * x);
    y = y - a * fnint(ra * y);
    z = z - a * fnint(ra * z);
  } else if (kImcon == 2) {
    x = x - c.h[0] * fnint(c.inv[0] * x);
    y = y - c.h[4] * fnint(c.inv[1] * y);
    z = z - c.h[8] * fnint(c.inv[2] * z);
  } else if (kImcon == 3) {
    const double* r = c.rh;
    double sx = r[0] * x + r[3] * y + r[6] * z;
    double sy = r[1] * x + r[4] * y + r[7] * z;
    double sz = r[2] * x + r[5] * y + r[8] * z;
    sx = sx - fnint(sx);
    sy = sy - fnint(sy);
    sz = sz - fnint(sz);
    x = c.h[0] * sx + c.h[3] * sy + c.h[6] * sz;
    y = c.h[1] * sx + c.h[4] * sy + c.h[7] * sz;
    z = c.h[2] * sx + c.h[5] * sy + c.h[8] * sz;
  } else if (kImcon == 4) {
    const double a = c.h[0], ra = c.inv[0];
    x = x - a * fnint(ra * x);
    y = y - a * fnint(ra * y);
    z = z - a * fnint(ra * z);
    if ((fabs(x) + fabs(y) + fabs(z)) >= (0.75 * a)) {
      x = x - 0.5 * copysign(fabs(a), x);
      y = y - 0.5 * copysign(fabs(a), y);
      z = z - 0.5 * copysign(fabs(a), z);
    }
  } else if (kImcon == 5) {
    const double a = c.h[0], cz = c.h[8];
    x = x - a * fnint(c.inv[0] * x);
    y = y - a * fnint(c.inv[0] * y);
    z = z - cz * fnint(c.inv[2] * z);
    if ((fabs(x) + fabs(y) + fabs(kImgRt2 * z)) >= a) {
      x = x - 0.5 * copysign(fabs(a), x);
      y = y - 0.5 * copysign(fabs(a), y);
      z = z - 0.5 * copysign(fabs(cz), z);
    }
  } else if (kImcon == 6) {  // periodic in the a-b plane only
    const double sx = c.slab[0] * x + c.slab[2] * y, sy = c.slab[1] * x + c.slab[3] * y;
    const double xss = sx - fnint(sx), yss = sy - fnint(sy);
    x = c.h[0] * xss + c.h[3] * yss;
    y = c.h[1] * xss + c.h[4] * yss;
  } else if (kImcon == 7) {
    const double aaa = c.hex[0], bbb = c.hex[1];
    y = y - bbb * fnint(c.hex[2] * y);
    z = z - c.h[8] * fnint(c.inv[2] * z);
    if ((fabs(y) + fabs(kImgRt3 * x)) >= bbb) {
      x = x - kImgRt3 * copysign(fabs(aaa), x);
      y = y - copysign(fabs(aaa), y);
    }
  }
}

// The same with the boundary condition read from the cell.
FMC_HD void min_image(const CellGeom& c, double& x, double& y, double& z) {
  if (c.imcon == 1) min_image_t<1>(c, x, y, z);
  else if (c.imcon == 2) min_image_t<2>(c, x, y, z);
  else if (c.imcon == 3) min_image_t<3>(c, x, y, z);
  else if (c.imcon == 4) min_image_t<4>(c, x, y, z);
  else if (c.imcon == 5) min_image_t<5>(c, x, y, z);
  else if (c.imcon == 6) min_image_t<6>(c, x, y, z);
  else if (c.imcon == 7) min_image_t<7>(c, x, y, z);
}

// Nearest in-plane image of a separation in a slab: the nint image and its eight neighbours in
// the a-b plane, z as it is.  A lower bound of the distance images() returns.
FMC_HD double slab_dist2(const CellGeom& c, double x, double y, double z) {
  min_image_t<6>(c, x, y, z);
  double best = 1e300;
  for (int i = -1; i <= 1; i++)
    for (int j = -1; j <= 1; j++) {
      const double u = x + i * c.h[0] + j * c.h[3], v = y + i * c.h[1] + j * c.h[4];
      best = fmin(best, u * u + v * v + z * z);
    }
  return best;
}

// Squared distance to the nearest lattice image of a separation: for imcon 4, 5 and 7 the
// lattice is the box's plus the box's shifted by half its a and b (and c for 4 and 5), so the
// nearest image is the nearer of the box-nearest images of the separation and of its shift.
// Builders of neighbour lists use it as a lower bound of the distance images() returns.
FMC_HD double shifted_lattice_dist2(const CellGeom& c, double x, double y, double z) {
  double best = 1e300;
  for (int k = 0; k < 2; k++) {
    double u = x + (k ? 0.5 * c.h[0] : 0.0), v = y + (k ? 0.5 * c.h[4] : 0.0);
    double w = z + (k && c.imcon != 7 ? 0.5 * c.h[8] : 0.0);
    u = u - c.h[0] * fnint(c.inv[0] * u);
    v = v - c.h[4] * fnint(c.inv[1] * v);
    w = w - c.h[8] * fnint(c.inv[2] * w);
    best = fmin(best, u * u + v * v + w * w);
  }
  return best;
}

// ------------------------------------------------------------------ trial generators
// rotation (utility_pack.f:2887-2926) of n sites by the quaternion q.
FMC_HD void rotate_sites(double* x, double* y, double* z, int n, const double q[4]) {
  const double q1 = q[0], q2 = q[1], q3 = q[2], q4 = q[3];
  const double Q0 = 2.0 * q2 * q2 + 2.0 * q1 * q1 - 1.0, Q1 = 2.0 * q2 * q3 - 2.0 * q1 * q4;
  const double Q2 = 2.0 * q2 * q4 + 2.0 * q1 * q3, Q3 = 2.0 * q2 * q3 + 2.0 * q1 * q4;
  const double Q4 = 2.0 * q1 * q1 + 2.0 * q3 * q3 - 1.0, Q5 = 2.0 * q3 * q4 - 2.0 * q1 * q2;
  const double Q6 = 2.0 * q2 * q4 - 2.0 * q1 * q3, Q7 = 2.0 * q3 * q4 + 2.0 * q1 * q2;
  const double Q8 = 2.0 * q4 * q4 + 2.0 * q1 * q1 - 1.0;
  for (int i = 0; i < n; i++) {
    double tx = Q0 * x[i] + Q1 * y[i] + Q2 * z[i];
    double ty = Q3 * x[i] + Q4 * y[i] + Q5 * z[i];
    double tz = Q6 * x[i] + Q7 * y[i] + Q8 * z[i];
    x[i] = tx;
    y[i] = ty;
    z[i] = tz;
  }
}

// Quaternion of angle theta about the axis (2r2-1, 2r3-1, 2r4-1)/norm (random_ins, random_rot).
FMC_HD void axis_angle_quat(double theta, double r2, double r3, double r4, double q[4]) {
  double b1 = 2.0 * r2 - 1.0, b2 = 2.0 * r3 - 1.0, b3 = 2.0 * r4 - 1.0;
  double st, ct;
  sincos(theta / 2.0, &st, &ct);
  double norm = sqrt(b1 * b1 + b2 * b2 + b3 * b3);
  q[0] = ct;
  q[1] = st * (b1 / norm);
  q[2] = st * (b2 / norm);
  q[3] = st * (b3 / norm);
}

// random_ins (utility_pack.f:2545-2650): template sites rotated by a random quaternion and
// placed with their COM at fractional (ra, rb, rc).
FMC_HD void trial_insert(const CellGeom& c, const double* tx, const double* ty, const double* tz, int n,
                         const double r[7], double* x, double* y, double* z) {
  const double* h = c.h;
  double xc = r[0] * h[0] + r[1] * h[3] + r[2] * h[6];
  double yc = r[0] * h[1] + r[1] * h[4] + r[2] * h[7];
  double zc = r[0] * h[2] + r[1] * h[5] + r[2] * h[8];
  for (int i = 0; i < n; i++) {
    x[i] = tx[i];
    y[i] = ty[i];
    z[i] = tz[i];
  }
  double q[4];
  axis_angle_quat(r[3] * 2.0 * kPi, r[4], r[5], r[6], q);
  rotate_sites(x, y, z, n, q);
  for (int i = 0; i < n; i++) {
    x[i] = x[i] + xc;
    y[i] = y[i] + yc;
    z[i] = z[i] + zc;
  }
}

// random_disp + random_rot (utility_pack.f:2679-2763, 2929-3000): translate by
// (2r-1)*delr/2 per Cartesian axis, wrap the mass COM into the cell, rotate about it.
FMC_HD void trial_displace(const CellGeom& c, const double* mass, int n, double delr, double rotangle,
                           const double r[7], double* x, double* y, double* z) {
  const double half = delr * 0.5;
  const double dx = (2.0 * r[0] - 1.0) * half, dy = (2.0 * r[1] - 1.0) * half, dz = (2.0 * r[2] - 1.0) * half;
  double w = 0.0, sx = 0.0, sy = 0.0, sz = 0.0;
  for (int i = 0; i < n; i++) {
    x[i] = dx + x[i];
    y[i] = dy + y[i];
    z[i] = dz + z[i];
  }
  for (int i = 0; i < n; i++) {
    w = w + mass[i];
    sx = sx + x[i] * mass[i];
    sy = sy + y[i] * mass[i];
    sz = sz + z[i] * mass[i];
  }
  double cx = sx / w, cy = sy / w, cz = sz / w;
  const double* rh = c.rh;
  const double* h = c.h;
  double fx = rh[0] * cx + rh[3] * cy + rh[6] * cz;
  double fy = rh[1] * cx + rh[4] * cy + rh[7] * cz;
  double fz = rh[2] * cx + rh[5] * cy + rh[8] * cz;
  fx = fx - floor(fx);
  fy = fy - floor(fy);
  fz = fz - floor(fz);
  double wx = h[0] * fx + h[3] * fy + h[6] * fz;
  double wy = h[1] * fx + h[4] * fy + h[7] * fz;
  double wz = h[2] * fx + h[5] * fy + h[8] * fz;
  double shx = wx - cx, shy = wy - cy, shz = wz - cz;
  for (int i = 0; i < n; i++) {
    x[i] = x[i] + shx - wx;
    y[i] = y[i] + shy - wy;
    z[i] = z[i] + shz - wz;
  }
  double q[4];
  axis_angle_quat(r[3] * rotangle, r[4], r[5], r[6], q);
  rotate_sites(x, y, z, n, q);
  for (int i = 0; i < n; i++) {
    x[i] = x[i] + wx;
    y[i] = y[i] + wy;
    z[i] = z[i] + wz;
  }
}

// energy_eval (utility_pack.f:3049-3095).  volm in m^3, press in Pa, eng in kcal/mol.
FMC_HD bool accept_move(double eng, double rande, double volm_m3, double press, int ngsts, double temp,
                        double beta, int move) {
  double test = 0.0;
  if (-1 * beta * eng > 700.0)
    test = exp(700.0);
  else if (move == kDisplace)
    test = exp(-1.0 * beta * eng);
  else if (move == kInsert)
    test = volm_m3 * press / ((ngsts + 1) * kBoltz * temp) * exp(-1.0 * beta * eng);
  else if (move == kDelete)
    test = fabs(press) < 1e-7 ? 1.0 : ngsts * kBoltz * temp / (volm_m3 * press) * exp(-1.0 * beta * eng);
  return rande < test;
}

// ------------------------------------------------------------------ probability plots
// One axis of equitable_bin (utility_pack.f:1880-1990): the two grid cells (0-based) whose
// centres bracket fractional position f on an n-cell axis, and their linear weights.
FMC_HD void equitable_axis(int n, double f, int& lo, int& hi, double& wl, double& wr) {
  double gp = n * f;
  int idx = (int)ceil(gp);
  double part = gp - floor(gp);
  if (part > 0.5) {
    lo = idx >= n ? n - 1 : idx - 1;
    hi = idx >= n ? 0 : idx;
    wl = 1.5 - part;
    wr = part - 0.5;
  } else {
    lo = idx <= 1 ? n - 1 : idx - 2;
    hi = idx <= 1 ? 0 : idx - 1;
    wl = 0.5 - part;
    wr = 0.5 + part;
  }
}

// The unit weight of fractional position (fa, fb, fc) spread over the 8 surrounding cells of an
// na x nb x nc grid (index a*nb*nc + b*nc + c), in the reference's order; add(index, weight).
template <class Add>
FMC_HD void equitable_bin(int na, int nb, int nc, double fa, double fb, double fc, Add add) {
  int al, ar, bl, br, cl, cr;
  double wal, war, wbl, wbr, wcl, wcr;
  equitable_axis(na, fa, al, ar, wal, war);
  equitable_axis(nb, fb, bl, br, wbl, wbr);
  equitable_axis(nc, fc, cl, cr, wcl, wcr);
  auto at = [&](int a, int b, int c) { return ((long long)a * nb + b) * nc + c; };
  add(at(al, bl, cl), wal * wbl * wcl);
  add(at(ar, bl, cl), war * wbl * wcl);
  add(at(al, br, cl), wal * wbr * wcl);
  add(at(al, bl, cr), wal * wbl * wcr);
  add(at(ar, br, cl), war * wbr * wcl);
  add(at(ar, bl, cr), war * wbl * wcr);
  add(at(al, br, cr), wal * wbr * wcr);
  add(at(ar, br, cr), war * wbr * wcr);
}

// Centre of mass of n sites (com, utility_pack.f:3003-3034); stride between sites' x values.
FMC_HD void centre_of_mass(const double* mass, int n, const double* x, const double* y, const double* z, int stride,
                           double* c) {
  double w = 0.0, sx = 0.0, sy = 0.0, sz = 0.0;
  for (int i = 0; i < n; i++) {
    w = w + mass[i];
    sx = sx + x[i * stride] * mass[i];
    sy = sy + y[i * stride] * mass[i];
    sz = sz + z[i * stride] * mass[i];
  }
  c[0] = sx / w;
  c[1] = sy / w;
  c[2] = sz / w;
}

// Fractional coordinates, wrapped into [0, 1) (frac / frac2, utility_pack.f:650-704).
FMC_HD void frac_wrap(const double* rh, double x, double y, double z, double* f) {
  double sx = x * rh[0] + y * rh[3] + z * rh[6];
  double sy = x * rh[1] + y * rh[4] + z * rh[7];
  double sz = x * rh[2] + y * rh[5] + z * rh[8];
  f[0] = sx - floor(sx);
  f[1] = sy - floor(sy);
  f[2] = sz - floor(sz);
}

// random_jump (utility_pack.f:2766-2813) + random_rot (2929-3000), rotangle = 8 atan(1): the
// centre of mass moves to fractional (r0, r1, r2) of the cell, then the molecule turns about it
// by r3 * 2 pi around the axis (2 r4 - 1, 2 r5 - 1, 2 r6 - 1).  x, y, z: current sites in,
// trial sites out.
FMC_HD void trial_jump(const CellGeom& c, const double* mass, int n, const double r[7], double* x, double* y,
                       double* z) {
  const double* h = c.h;
  double xd = r[0] * h[0] + r[1] * h[3] + r[2] * h[6];
  double yd = r[0] * h[1] + r[1] * h[4] + r[2] * h[7];
  double zd = r[0] * h[2] + r[1] * h[5] + r[2] * h[8];
  double cm[3];
  centre_of_mass(mass, n, x, y, z, 1, cm);
  xd = xd - cm[0];
  yd = yd - cm[1];
  zd = zd - cm[2];
  for (int i = 0; i < n; i++) {
    x[i] = xd + x[i];
    y[i] = yd + y[i];
    z[i] = zd + z[i];
  }
  centre_of_mass(mass, n, x, y, z, 1, cm);
  for (int i = 0; i < n; i++) {
    x[i] = x[i] - cm[0];
    y[i] = y[i] - cm[1];
    z[i] = z[i] - cm[2];
  }
  double q[4];
  axis_angle_quat(r[3] * (8.0 * atan(1.0)), r[4], r[5], r[6], q);
  rotate_sites(x, y, z, n, q);
  for (int i = 0; i < n; i++) {
    x[i] = x[i] + cm[0];
    y[i] = y[i] + cm[1];
    z[i] = z[i] + cm[2];
  }
}

// ------------------------------------------------------------------ windowed statistics
constexpr double kRgas = 8.314472 / 4184.0;  // kcal/mol/K (utility_pack.f:109)
constexpr int kSampleCap = 500000;           // stored production samples per species (gcmc.f)

// calc_Qst and calc_Cv (utility_pack.f:2280-2316)
FMC_HD double calc_qst(double E2, double E, double N, double N2, double EN, double temp) {
  (void)E2;
  return -1.0 * (EN - E * N) / (N2 - N * N) + kRgas * temp;
}
FMC_HD double calc_cv(double E2, double E, double N, double N2, double EN, double temp) {
  const double d = EN - E * N;
  return (3.0 / 2.0 * kRgas) + (E2 - (E * E) - d * d / (N2 - N * N)) / (N * kKboltz * temp * temp);
}

// The reference's averaging windows (gcmc.f:1814-1928): rolling window means of N, E, EN, N^2,
// E^2 (and <exp(-dE/kT)> of insertions), closed every `nwind` production samples into weighted
// running means and variances, with the selectivities between species.
// Pressure equilibration (gcmc.f:649-693), at a 400-move check: the partial pressures are
// redistributed from the target loadings (adsguen), the running loading since the last
// adjustment (read and cleared through nmean, `stride` doubles apart) and the ideal-gas term of
// the free volume, then rescaled to the same total; the tolerance and the move count are cleared
// once the last species' rate falls under it or the move count passes -50 * eqsteps.  The
// reference indexes these arrays by FIELD molecule index, so guests come first in FIELD.
FMC_HD void pressure_adjust(int ng, double* press, double* nmean, int stride, const double* adspres,
                            const double* adsguen, double packf, double volm, double temp, double& presrate,
                            double& despre, int& gcmccount, long long& prodcount, int eqsteps) {
  double totpres = 0.0;
  for (int i = 0; i < ng; i++) totpres += press[i];
  double dqp[kMaxGuestTypes];
  for (int i = 0; i < ng; i++) {
    const double temppres = (press[i] * (1 - packf) * volm / packf) / (temp * 13806874.7924278);
    dqp[i] = adsguen[i] - nmean[i * stride] + (adspres[i] - temppres);
    nmean[i * stride] = 0;
  }
  double presleft = 0.0;
  for (int i = 0; i < ng - 1; i++) {
    double sd = 0.0;
    for (int k = 0; k < ng; k++) sd += dqp[k];
    presrate = dqp[i] - sd * press[i] / totpres;
    press[i] = dqp[i] * totpres / sd;
    if (press[i] < 0) press[i] = 0;
    presleft = presleft + press[i];
  }
  press[ng - 1] = totpres - presleft;
  if (press[ng - 1] < 0) press[ng - 1] = 0;
  double sp = 0.0;
  for (int i = 0; i < ng; i++) sp += press[i];
  const double changerate = totpres / sp;
  for (int i = 0; i < ng; i++) press[i] = press[i] * changerate;
  prodcount = 0;
  if (fabs(presrate) < despre || (long long)gcmccount > -50LL * eqsteps) {
    gcmccount = 0;
    despre = 0;
  }
}

struct WindowStats {
  int rollcount, ins_rollcount, avcount;
  double avg[kMaxGuestTypes][8], sum[kMaxGuestTypes][8], var[kMaxGuestTypes][8];
  double seltot[kMaxGuestTypes][kMaxGuestTypes], selwin[kMaxGuestTypes][kMaxGuestTypes];
};

// One counted production sample of species i, after its cumulative averages cs[0..4] (<N>,
// <E>, <EN>, <N^2>, <E^2>) were updated; cs[5] is the rolling <exp(-dE/kT)> of accepted
// insertions.  rollcount must already count this sample.
FMC_HD void window_sample(WindowStats& W, int i, double dm, double e, bool ins_accepted, double delE, double temp,
                          int accept_ins, double* cs) {
  double* aw = W.avg[i];
  if (ins_accepted) {
    double h = exp(-1.0 * delE / kKboltz / temp);
    W.ins_rollcount++;
    double delta = h - cs[5];
    h = cs[5] + delta / accept_ins;
    cs[5] = h;
    aw[7] = ((W.ins_rollcount - 1) * aw[7] + h) / (double)W.ins_rollcount;
  }
  const double rc = (double)W.rollcount;
  aw[0] = ((W.rollcount - 1) * aw[0] + dm) / rc;
  aw[1] = ((W.rollcount - 1) * aw[1] + e) / rc;
  aw[2] = ((W.rollcount - 1) * aw[2] + e * dm) / rc;
  aw[3] = ((W.rollcount - 1) * aw[3] + dm * dm) / rc;
  aw[4] = ((W.rollcount - 1) * aw[4] + e * e) / rc;
}

// Closes a window (gcmc.f:1887-1928); cs(i) gives species i's cumulative averages.
template <class CS>
FMC_HD void window_close(WindowStats& W, int ng, int nwind, double temp, CS cs) {
  W.avcount++;
  const double weight = (double)W.rollcount / (double)nwind;
  for (int i = 0; i < ng; i++) {
    const double* c = cs(i);
    double* aw = W.avg[i];
    aw[5] = calc_qst(c[4], c[1], c[0], c[3], c[2], temp);
    aw[6] = calc_cv(c[4], c[1], c[0], c[3], c[2], temp);
    if (i > 0) {
      const double an = aw[0];
      for (int j = 0; j < i; j++) {
        if (an == 0) continue;
        const double sel = W.avg[j][0] / an;
        const double delta = weight * (sel - W.seltot[i][j]);
        W.seltot[i][j] = W.seltot[i][j] + delta / W.avcount;
        W.selwin[i][j] = W.selwin[i][j] + weight * (sel * sel - W.selwin[i][j]) / (W.avcount - 1 + weight);
        W.seltot[j][i] = ((W.avcount - 1 + weight) * W.selwin[i][j] -
                          ((W.avcount - 1 + weight) * W.seltot[i][j] * W.seltot[i][j])) /
                         (W.avcount - 1 + weight);
      }
    }
  }
  for (int i = 0; i < ng; i++)
    for (int k = 0; k < 8; k++) {
      const double delta = weight * (W.avg[i][k] - W.sum[i][k]);
      W.sum[i][k] = W.sum[i][k] + delta / W.avcount;
      W.var[i][k] = W.var[i][k] + delta * weight * (W.avg[i][k] - W.sum[i][k]);
      W.avg[i][k] = 0.0;
    }
  W.rollcount = 0;
}

// 3-point interpolation of a tabulated function on r_l = l*dr (ewald.f:670-684,
// vdw_terms.f:476-489).  tab[0] is defined as tab[1].
FMC_HD double interp3(const double* tab, double rrr, double rdr) {
  int l = (int)(rrr * rdr);
  double ppp = rrr * rdr - (double)l;
  double v0 = tab[l], v1 = tab[l + 1], v2 = tab[l + 2];
  double t1 = v0 + (v1 - v0) * ppp;
  double t2 = v1 + (v2 - v1) * (ppp - 1.0);
  return t1 + (t2 - t1) * ppp * 0.5;
}

}  // namespace fmc
