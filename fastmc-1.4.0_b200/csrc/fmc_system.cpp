// Host-side system builder: tables, k-vectors, LRC terms, guest constants, voxel lists.
#include "fmc_system.h"

#include <algorithm>
#include <cmath>

namespace fmc {
namespace {

void invert3(const double* a, double* b) {
  // invert, utility_pack.f:1417-1467 (adjoint / determinant)
  b[0] = a[4] * a[8] - a[5] * a[7];
  b[1] = a[2] * a[7] - a[1] * a[8];
  b[2] = a[1] * a[5] - a[2] * a[4];
  b[3] = a[5] * a[6] - a[3] * a[8];
  b[4] = a[0] * a[8] - a[2] * a[6];
  b[5] = a[2] * a[3] - a[0] * a[5];
  b[6] = a[3] * a[7] - a[4] * a[6];
  b[7] = a[1] * a[6] - a[0] * a[7];
  b[8] = a[0] * a[4] - a[1] * a[3];
  double d = a[0] * b[0] + a[3] * b[1] + a[6] * b[2];
  double r = std::fabs(d) > 0.0 ? 1.0 / d : 0.0;
  for (int i = 0; i < 9; i++) b[i] = r * b[i];
}

// perpendicular widths of a cell (dcell bbb(7..9))
void widths(const double* a, double* w) {
  double axb[3] = {a[1] * a[5] - a[2] * a[4], a[2] * a[3] - a[0] * a[5], a[0] * a[4] - a[1] * a[3]};
  double bxc[3] = {a[4] * a[8] - a[5] * a[7], a[5] * a[6] - a[3] * a[8], a[3] * a[7] - a[4] * a[6]};
  double cxa[3] = {a[7] * a[2] - a[1] * a[8], a[0] * a[8] - a[2] * a[6], a[1] * a[6] - a[0] * a[7]};
  double v = std::fabs(a[0] * bxc[0] + a[1] * bxc[1] + a[2] * bxc[2]);
  w[0] = v / std::sqrt(bxc[0] * bxc[0] + bxc[1] * bxc[1] + bxc[2] * bxc[2]);
  w[1] = v / std::sqrt(cxa[0] * cxa[0] + cxa[1] * cxa[1] + cxa[2] * cxa[2]);
  w[2] = v / std::sqrt(axb[0] * axb[0] + axb[1] * axb[1] + axb[2] * axb[2]);
}

double ipow(double x, int m) {
  unsigned n = (unsigned)m;
  double y = (n & 1) ? x : 1.0;
  while (n >>= 1) {
    x = x * x;
    if (n & 1) y = y * x;
  }
  return y;
}

// One tabulated potential value (forgen, vdw_terms.f:189-396)
double vdw_value(int key, const std::array<double, 5>& p, double rrr, double rvdw) {
  switch (key) {
    case 1:
      return (p[0] / ipow(rrr, 6) - p[1]) / ipow(rrr, 6);
    case 2: {
      double sr = p[1] / rrr;
      return 4.0 * p[0] * ipow(sr, 6) * (ipow(sr, 6) - 1.0);
    }
    case 3: {
      double ann = std::max(p[1], p[2]), amm = std::min(p[1], p[2]);
      return p[0] / (ann - amm) * (amm * std::pow(p[3] / rrr, ann) - ann * std::pow(p[3] / rrr, amm));
    }
    case 4:
      return p[0] * std::exp(-rrr / p[1]) - p[2] / ipow(rrr, 6);
    case 5:
      return p[0] * std::exp(p[1] * (p[2] - rrr)) - p[3] / ipow(rrr, 6) - p[4] / ipow(rrr, 8);
    case 6:
      return p[0] / ipow(rrr, 12) - p[1] / ipow(rrr, 10);
    case 7: {
      double eps = p[0], ann = p[1], amm = p[2], rr0 = p[3], rrc = p[4];
      if (rrc < 1e-6) rrc = rvdw;
      double gam = rrc / rr0;
      double bet = gam * std::pow((std::pow(gam, amm + 1.0) - 1.0) / (std::pow(gam, ann + 1.0) - 1.0), 1.0 / (ann - amm));
      eps = -eps * (ann - amm) /
            (amm * std::pow(bet, ann) * (1.0 + (ann / gam - ann - 1.0) / std::pow(gam, ann)) -
             ann * std::pow(bet, amm) * (1.0 + (amm / gam - amm - 1.0) / std::pow(gam, amm)));
      if (rrr > rrc) return 0.0;
      return eps / (ann - amm) *
             (amm * std::pow(bet, ann) * (std::pow(rr0 / rrr, ann) - std::pow(1.0 / gam, ann)) -
              ann * std::pow(bet, amm) * (std::pow(rr0 / rrr, amm) - std::pow(1.0 / gam, amm)) +
              ann * amm * ((rrr / (gam * rr0) - 1.0) * (std::pow(bet / gam, ann) - std::pow(bet / gam, amm))));
    }
    case 8: {
      double t = 1.0 - std::exp(-p[2] * (rrr - p[1]));
      return p[0] * (t * t - 1.0);
    }
    case 9: {
      double ddd = p[1] * std::pow(2.0, 1.0 / 6.0);
      double rr = rrr - p[2];
      if (rr > ddd) return 0.0;
      if (rr > 0.0) {
        double sr = p[1] / rr;
        return 4.0 * p[0] * ipow(sr, 6) * (ipow(sr, 6) - 1.0) + p[0];
      }
      return 0.0;
    }
    default:
      return 0.0;
  }
}

// Tail-correction pair term (lrcorrect eadd, vdw_terms.f:581-650)
double lrc_eadd(int key, const std::array<double, 5>& p, double rcut) {
  switch (key) {
    case 0:
      return p[0];
    case 1:
      return p[0] / (9.0 * ipow(rcut, 9)) - p[1] / (3.0 * ipow(rcut, 3));
    case 2:
      return 4.0 * p[0] * (ipow(p[1], 12) / (9.0 * ipow(rcut, 9)) - ipow(p[1], 6) / (3.0 * ipow(rcut, 3)));
    case 3: {
      double eps = p[0], ann = p[1], amm = p[2], rr0 = p[3];
      return eps / (ann - amm) *
             (amm * std::pow(rr0, ann) / ((ann - 3.0) * std::pow(rcut, ann - 3.0)) -
              ann * std::pow(rr0, amm) / ((amm - 3.0) * std::pow(rcut, amm - 3.0)));
    }
    case 4:
      return -p[2] / (3.0 * ipow(rcut, 3));
    case 5:
      return -p[3] / (3.0 * ipow(rcut, 3)) - p[4] / (5.0 * ipow(rcut, 5));
    case 6:
      return p[0] / (9.0 * ipow(rcut, 9)) - p[1] / (7.0 * ipow(rcut, 7));
    default:
      return 0.0;
  }
}

// True minimum-image distance^2 (the nint image and its 26 neighbours).
double true_dist2(const CellGeom& c, double dx, double dy, double dz) {
  if (c.imcon == 4 || c.imcon == 5 || c.imcon == 7) return shifted_lattice_dist2(c, dx, dy, dz);
  if (c.imcon == 6) return slab_dist2(c, dx, dy, dz);
  min_image(c, dx, dy, dz);
  if (c.imcon == 1 || c.imcon == 2) return dx * dx + dy * dy + dz * dz;
  double best = dx * dx + dy * dy + dz * dz;
  for (int i = -1; i <= 1; i++)
    for (int j = -1; j <= 1; j++)
      for (int k = -1; k <= 1; k++) {
        double x = dx + i * c.h[0] + j * c.h[3] + k * c.h[6];
        double y = dy + i * c.h[1] + j * c.h[4] + k * c.h[7];
        double z = dz + i * c.h[2] + j * c.h[5] + k * c.h[8];
        best = std::min(best, x * x + y * y + z * z);
      }
  return best;
}

}  // namespace

double ewald3_pair(double alpha, double chgprd, double rrr) {
  const double a1 = 0.254829592, a2 = -0.284496736, a3 = 1.421413741;
  const double a4 = -1.453152027, a5 = 1.061405429, pp = 0.3275911;
  const double rr3 = 0.333333333333, r10 = 0.1, r42 = 0.02380952381, r216 = 4.62962962963e-3;
  double alpr = rrr * alpha, alpr2 = alpr * alpr;
  if (alpr < 1e-2)
    return 2.0 * chgprd * (alpha / kSqrPi) * (1.0 + alpr2 * (-rr3 + alpr2 * (r10 + alpr2 * (-r42 + alpr2 * r216))));
  double tt = 1.0 / (1.0 + pp * alpha * rrr);
  double ar = alpha * rrr;
  double e1 = std::exp(-(ar * ar));
  return (1.0 - tt * (a1 + tt * (a2 + tt * (a3 + tt * (a4 + tt * a5)))) * e1) * chgprd / rrr;
}

double lrc_energy(const HostSystem& s, const std::vector<int>& numtyp, const std::vector<int>& numfrz) {
  if (!s.lrc_on) return 0.0;
  const double twopi = 2.0 * kPi, v = s.cell.volm;
  double e = 0.0;
  int ivdw = 0;
  for (int i = 1; i <= s.ntypes; i++)
    for (int j = 1; j <= i; j++) {
      ivdw++;
      double den = twopi * ((double)numtyp[i] * (double)numtyp[j] - (double)numfrz[i] * (double)numfrz[j]) / (v * v);
      e = e + v * den * s.steadd[ivdw];
    }
  return e;
}

int build_host_system(const InputDeck& d, HostSystem& s, std::string& err, double voxel_edge) {
  s = HostSystem();
  s.deck = d;
  if (d.imcon < 1 || d.imcon > 7) {
    err = "cells without periodic boundaries (imcon 0) are not supported on the device";
    return -4;
  }
  // ---- cell
  for (int i = 0; i < 9; i++) s.cell.h[i] = d.cell[i];
  invert3(d.cell, s.cell.rh);
  cell_reciprocals(s.cell);
  s.cell.volm = d.volm;
  s.cell.imcon = d.imcon;
  s.rcut = d.rcut;
  s.alpha = d.alpha;
  s.engunit = d.engunit;
  s.beta = 1.0 / (kKboltz * d.temp);
  s.statvolm = d.volm * 1e-30;
  s.mxgrid = d.mxgrid;
  // ---- erc table (erfcgen, ewald.f:1-30)
  {
    const double a1 = 0.254829592, a2 = -0.284496736, a3 = 1.421413741;
    const double a4 = -1.453152027, a5 = 1.061405429, pp = 0.3275911;
    s.erc.assign(s.mxgrid + 1, 0.0);
    s.drewd = d.rcut / (double)(s.mxgrid - 4);
    for (int i = 1; i <= s.mxgrid; i++) {
      double rrr = (double)i * s.drewd;
      double tt = 1.0 / (1.0 + pp * d.alpha * rrr);
      double ar = d.alpha * rrr;
      double e1 = std::exp(-(ar * ar));
      s.erc[i] = tt * (a1 + tt * (a2 + tt * (a3 + tt * (a4 + tt * a5)))) * e1 / rrr;
    }
    s.erc[0] = s.erc[1];
  }
  // ---- vdW tables (forgen) incl. the zero table for undefined pairs
  s.ntypes = (int)d.types.size();
  if (s.ntypes > 255) {
    err = "more than 255 unique atom types";
    return -5;
  }
  s.ntables = d.ntpvdw + 1;
  s.dlrpot = d.rvdw / (double)(s.mxgrid - 4);
  const int stride = s.mxgrid + 1;
  s.vvv.assign((size_t)(s.ntables + 1) * stride, 0.0);
  for (int k = 1; k <= d.ntpvdw; k++) {
    double* row = &s.vvv[(size_t)k * stride];
    for (int i = 1; i <= s.mxgrid; i++) row[i] = vdw_value(d.ltpvdw[k], d.prmvdw[k], (double)i * s.dlrpot, d.rvdw);
    row[0] = row[1];
  }
  s.pair_row.assign((s.ntypes + 1) * (s.ntypes + 1), -1);
  for (int a = 1; a <= s.ntypes; a++)
    for (int b = 1; b <= s.ntypes; b++) {
      int hi = std::max(a, b), lo = std::min(a, b);
      int k = d.lstvdw[hi * (hi - 1) / 2 + lo];
      if (k < 1 || k > s.ntables) continue;
      int key = d.ltpvdw[k];
      double v1 = s.vvv[(size_t)k * stride + 1];
      // srfrce skips pairs whose table is a placeholder or vanishes (vdw_terms.f:467)
      if (key < 100 && std::fabs(v1) > 1e-10) s.pair_row[a * (s.ntypes + 1) + b] = k;
    }
  // ---- k-vectors in the reference's half-space order (ewald.f:77-84, 139-331)
  {
    const double twopi = 2.0 * kPi;
    const double* rc = s.cell.rh;
    double w[3];
    widths(rc, w);
    double rcpcut = std::min(std::min((double)d.kmax[0] * w[0], (double)d.kmax[1] * w[1]), (double)d.kmax[2] * w[2]);
    rcpcut = rcpcut * 1.05 * twopi;
    double rcpct2 = rcpcut * rcpcut;
    bool lconsw = !(d.imcon == 4 || d.imcon == 5 || d.imcon == 7);
    double ralph = -0.25 / (d.alpha * d.alpha);
    int mmin = 0, nmin = 1;
    for (int ll = 0; ll <= d.kmax[0]; ll++) {
      double t1 = twopi * (double)ll;
      double rkx1 = t1 * rc[0], rky1 = t1 * rc[3], rkz1 = t1 * rc[6];
      for (int mm = mmin; mm <= d.kmax[1]; mm++) {
        double t2 = twopi * (double)mm;
        double rkx2 = rkx1 + t2 * rc[1], rky2 = rky1 + t2 * rc[4], rkz2 = rkz1 + t2 * rc[7];
        for (int nn = nmin; nn <= d.kmax[2]; nn++) {
          double t3 = twopi * (double)nn;
          double rkx3 = rkx2 + t3 * rc[2], rky3 = rky2 + t3 * rc[5], rkz3 = rkz2 + t3 * rc[8];
          double rksq = rkx3 * rkx3 + rky3 * rky3 + rkz3 * rkz3;
          if (rksq <= rcpct2) {
            double rr = 1.0 / rksq;
            double a = std::exp(ralph * rksq) * rr;
            if (!lconsw) a = 4.0 * std::exp(ralph * rksq) * rr;
            s.kl.push_back(ll);
            s.km.push_back(mm);
            s.kn.push_back(nn);
            s.akk.push_back(a);
          }
        }
        nmin = -d.kmax[2];
      }
      mmin = -d.kmax[1];
    }
    s.K = (int)s.akk.size();
    double rvolm = twopi / d.volm;
    s.recip_pref = lconsw ? 2.0 * rvolm * kR4pie0 : 0.5 * rvolm * kR4pie0;
  }
  // ---- long-range correction terms (lrcorrect steadd, vdw_terms.f:564-672)
  s.lrc_on = (d.imcon != 0 && d.imcon != 6 && d.maxvdw > 0 && d.keyfce % 2 == 0);
  {
    int ntab = s.ntypes * (s.ntypes + 1) / 2;
    s.steadd.assign(ntab + 1, 0.0);
    int ivdw = 0;
    for (int i = 1; i <= s.ntypes; i++)
      for (int j = 1; j <= i; j++) {
        ivdw++;
        int k = d.lstvdw[ivdw];
        double e = (k >= 1 && k <= d.ntpvdw) ? lrc_eadd(d.ltpvdw[k], d.prmvdw[k], d.rcut) : 0.0;
        if (i != j) e = e * 2.0;
        s.steadd[ivdw] = e;
      }
  }
  // ---- per-guest constants
  const int ng = (int)d.guests.size();
  s.engsic.assign(ng, 0.0);
  s.ewald3en.assign(ng, 0.0);
  s.mvcum.assign(ng, {});
  for (int g = 0; g < ng; g++) {
    const GuestSpecies& G = d.guests[g];
    double q2 = 0.0;
    for (int i = 0; i < G.nsite; i++) q2 = q2 + G.charge[i] * G.charge[i];
    s.engsic[g] = -kR4pie0 * d.alpha * q2 / kSqrPi;
    double e3 = 0.0;
    for (int i = 0; i < G.nsite - 1; i++) {
      double part = 0.0, chgea = G.charge[i] * kR4pie0;
      for (int j = i + 1; j < G.nsite; j++) {
        double dx = G.tx[i] - G.tx[j], dy = G.ty[i] - G.ty[j], dz = G.tz[i] - G.tz[j];
        min_image(s.cell, dx, dy, dz);
        double r = std::sqrt(dx * dx + dy * dy + dz * dz);
        part = part - ewald3_pair(d.alpha, chgea * G.charge[j], r);
      }
      e3 = e3 + part;
    }
    s.ewald3en[g] = e3;
    // move-frequency normalisation (gcmc.f:282-331)
    std::array<double, 9> f = d.movefreq[g];
    double nrm = 0;
    for (double v : f) nrm += v;
    if (nrm == 0) {
      nrm = 1;
      f = {1.0 / 3.0, 1.0 / 3.0, 1.0 / 3.0, 0, 0, 0, 0, 0, 0};
    }
    std::array<double, 9> c;
    c[0] = f[0] / nrm;
    for (int k = 1; k < 9; k++) c[k] = c[k - 1] + (f[k] / nrm);
    s.mvcum[g] = c;
  }
  // ---- framework
  s.nf = (int)d.fq.size();
  s.fx = d.fx;
  s.fy = d.fy;
  s.fz = d.fz;
  s.fq = d.fq;
  s.ftype = d.ftype;
  s.ffrz = d.ffrz;
  // ---- voxel grid over the framework (lists are built on the device)
  {
    double w[3];
    widths(s.cell.h, w);
    for (int a = 0; a < 3; a++) s.nvox[a] = std::max(1, (int)std::floor(w[a] / voxel_edge));
    double e[3][3];
    for (int a = 0; a < 3; a++)
      for (int k = 0; k < 3; k++) e[a][k] = s.cell.h[3 * a + k] / s.nvox[a];
    if (d.imcon == 6) {
      // slab: layers of height voxel_edge along z over the framework's z range, widened by one
      // layer beyond the list radius at each end so that the end layers hold no atom and a
      // position beyond them can be clamped into them
      double zmin = 0.0, zmax = 0.0;
      for (int j = 0; j < (int)d.fz.size(); j++) {
        zmin = j ? std::min(zmin, d.fz[j]) : d.fz[j];
        zmax = j ? std::max(zmax, d.fz[j]) : d.fz[j];
      }
      e[2][0] = e[2][1] = 0.0;
      e[2][2] = voxel_edge;
      double circ6 = 0.0;
      for (int sa = -1; sa <= 1; sa += 2)
        for (int sb = -1; sb <= 1; sb += 2) {
          double v[3];
          for (int k = 0; k < 3; k++) v[k] = e[0][k] + sa * e[1][k] + sb * e[2][k];
          circ6 = std::max(circ6, 0.5 * std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]));
        }
      const double reach = s.rcut + circ6 + 1.0;  // the list radius, with room for the guest extent
      s.cell.dz = voxel_edge;
      s.cell.rdz = 1.0 / voxel_edge;
      s.cell.zlo = zmin - reach - voxel_edge;
      s.nvox[2] = (int)std::ceil((zmax - zmin + 2.0 * (reach + voxel_edge)) / voxel_edge);
    }
    double circ = 0.0;
    for (int sa = -1; sa <= 1; sa += 2)
      for (int sb = -1; sb <= 1; sb += 2) {
        double v[3];
        for (int k = 0; k < 3; k++) v[k] = e[0][k] + sa * e[1][k] + sb * e[2][k];
        circ = std::max(circ, 0.5 * std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]));
      }
    double lim = s.rcut + circ + 1e-6;
    s.vox_lim2 = lim * lim;
  }
  return 0;
}

void build_host_voxels(HostSystem& s) {
  int nv = s.nvox[0] * s.nvox[1] * s.nvox[2];
  s.vox_off.assign(nv + 1, 0);
  s.vox_atoms.clear();
  const double* h = s.cell.h;
  for (int a = 0; a < s.nvox[0]; a++)
    for (int b = 0; b < s.nvox[1]; b++)
      for (int c = 0; c < s.nvox[2]; c++) {
        double fa = (a + 0.5) / s.nvox[0], fb = (b + 0.5) / s.nvox[1], fc = (c + 0.5) / s.nvox[2];
        double cx = fa * h[0] + fb * h[3] + fc * h[6];
        double cy = fa * h[1] + fb * h[4] + fc * h[7];
        double cz = fa * h[2] + fb * h[5] + fc * h[8];
        if (s.cell.imcon == 6) {  // slab: in-plane cell, z layers from zlo
          cx = fa * h[0] + fb * h[3];
          cy = fa * h[1] + fb * h[4];
          cz = s.cell.zlo + (c + 0.5) * s.cell.dz;
        }
        int v = (a * s.nvox[1] + b) * s.nvox[2] + c;
        for (int j = 0; j < s.nf; j++)
          if (true_dist2(s.cell, cx - s.fx[j], cy - s.fy[j], cz - s.fz[j]) < s.vox_lim2) s.vox_atoms.push_back(j);
        s.vox_off[v + 1] = (int)s.vox_atoms.size();
      }
  s.vox_entries = (long long)s.vox_atoms.size();
}

}  // namespace fmc
