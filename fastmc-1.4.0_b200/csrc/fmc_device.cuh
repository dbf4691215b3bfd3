// Device-resident views of a GCMC system and of one chain's mutable state, plus the
// block-level building blocks shared by the plain (one launch per trial) kernels and the
// persistent batched kernel.
//
// HBM layout (per system, immutable): framework atoms as double4 {x,y,z,q} in condensed
// order + int type; voxel lists (CSR, ascending atom index); erc/vvv tables (mxgrid+1 doubles
// per row); k-vector table packed (l | (m+128)<<8 | (n+128)<<16) + akk (double).
// Per chain (mutable): S(k) as double2 {Re, Im}; guest sites as double4 {x,y,z,q} + int type,
// one contiguous segment per guest species, molecules in the reference's order.
#pragma once
#include <cuda_runtime.h>

#include "fmc_common.h"

namespace fmc {

struct DevSystem {
  CellGeom cell;
  int nf;
  const double4* fw;
  const int* fw_type;
  int nvox[3];
  const int* vox_off;
  const int* vox_atoms;
  const unsigned short* vox_atoms16;  // the same lists as 16-bit indices (null when nf > 65535)
  const double4* vox_xyzq;            // the same lists with each entry's atom inlined, and
  const unsigned char* vox_type;      // its type (coalesced one-hop reads)
  double rcut2, rdr_e, rdr_v;
  const double* erc;
  const double* vvv;
  int tab_stride;
  int ntypes;
  const int* pair_row;
  int K;
  int kmax[3];
  const int* kpack;
  const double* akk;
  double recip_pref;
};

constexpr int kMaxPassSites = 2 * kMaxGuestSites;

// Guest-site segments of one chain as seen by one launch (counts passed by value).
struct GuestView {
  const double4* site;
  const int* type;
  int nseg;
  int seg_off[kMaxGuestTypes];
  int seg_len[kMaxGuestTypes];  // sites currently present
};

FMC_HD int kpack(int l, int m, int n) { return l | ((m + 128) << 8) | ((n + 128) << 16); }
FMC_HD void kunpack(int p, int& l, int& m, int& n) {
  l = p & 0xff;
  m = ((p >> 8) & 0xff) - 128;
  n = ((p >> 16) & 0xff) - 128;
}

#if defined(__CUDACC__)

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.y * b.x + b.y * a.x);
}
__device__ __forceinline__ double2 cmulc(double2 a, double2 b) {  // a * conj(b)
  return make_double2(a.x * b.x + a.y * b.y, a.y * b.x - b.y * a.x);
}

// e^{i 2 pi j s} for j = 0..kmax by the recurrence of ewald.f:118-137 into tab[0..kmax].
__device__ __forceinline__ void axis_phases(double s, int kmax, double2* tab) {
  double sn, cs;
  sincos(2.0 * kPi * s, &sn, &cs);
  tab[0] = make_double2(1.0, 0.0);
  if (kmax >= 1) tab[1] = make_double2(cs, sn);
  for (int j = 2; j <= kmax; j++) {
    double2 p = tab[j - 1];
    tab[j] = make_double2(p.x * cs - p.y * sn, p.y * cs + p.x * sn);
  }
}

// Fractional coordinates s = rcell . r as in ewald.f:106-108.
__device__ __forceinline__ void frac_coords(const CellGeom& c, double x, double y, double z, double* s) {
  const double* r = c.rh;
  s[0] = r[0] * x + r[3] * y + r[6] * z;
  s[1] = r[1] * x + r[4] * y + r[7] * z;
  s[2] = r[2] * x + r[5] * y + r[8] * z;
}

// Pair energy of one site with charge factor chgea = q_i*r4pie0 and table row lookup base.
// kImcon < 0: the boundary condition is read from the cell.
template <int kImcon = -1>
__device__ __forceinline__ void pair_energy(const DevSystem& S, double dx, double dy, double dz, double chgea,
                                            double qj, int row, double& ec, double& ev) {
  if (kImcon < 0) min_image(S.cell, dx, dy, dz);
  else min_image_t<kImcon>(S.cell, dx, dy, dz);
  double rsq = dx * dx + dy * dy + dz * dz;
  if (rsq < S.rcut2) {
    double r = sqrt(rsq);
    double chgprd = chgea * qj;
    if (fabs(chgprd) > 1e-10) ec += interp3(S.erc, r, S.rdr_e) * chgprd;
    if (row >= 0) ev += interp3(S.vvv + (size_t)row * S.tab_stride, r, S.rdr_v);
  }
}

// Voxel of a position (wrapped into the cell; a slab's z clamped to its layers, whose lowest and
// highest hold no atom).
__device__ __forceinline__ int voxel_of(const DevSystem& S, double x, double y, double z) {
  double s[3];
  if (S.cell.imcon == 6) {
    const CellGeom& c = S.cell;
    s[0] = c.slab[0] * x + c.slab[2] * y;
    s[1] = c.slab[1] * x + c.slab[3] * y;
    s[2] = 0.0;
    double t = (z - c.zlo) * c.rdz;
    int k = t < 0.0 ? 0 : (t >= (double)S.nvox[2] ? S.nvox[2] - 1 : (int)t);
    int v0 = (int)((s[0] - floor(s[0])) * S.nvox[0]), v1 = (int)((s[1] - floor(s[1])) * S.nvox[1]);
    v0 = v0 < 0 ? 0 : (v0 >= S.nvox[0] ? S.nvox[0] - 1 : v0);
    v1 = v1 < 0 ? 0 : (v1 >= S.nvox[1] ? S.nvox[1] - 1 : v1);
    return (v0 * S.nvox[1] + v1) * S.nvox[2] + k;
  }
  frac_coords(S.cell, x, y, z, s);
  int v[3];
  for (int a = 0; a < 3; a++) {
    double f = s[a] - floor(s[a]);
    int i = (int)(f * S.nvox[a]);
    v[a] = i < 0 ? 0 : (i >= S.nvox[a] ? S.nvox[a] - 1 : i);
  }
  return (v[0] * S.nvox[1] + v[1]) * S.nvox[2] + v[2];
}

// A guest-site update accepted on the host and not yet written to the device arrays (an
// insert appends a molecule to its species' segment, a delete removes one and shifts the rest
// down, a displacement overwrites one).  The next trial pass reads the guest sites as if the
// update were written (GuestView indices are those after it) and writes it once every block of
// that pass has read them.
constexpr int kMaxPendSites = 8;
struct PendingCommit {
  int op;       // 0: none; kInsert, kDelete, kDisplace
  int seg;      // species segment index (-1: none)
  int lo;       // first site of the molecule (insert: the segment's end before the insert)
  int ns;       // sites per molecule
  int seg_end;  // end of the segment before the update
  double4 site[kMaxPendSites];
  int type[kMaxPendSites];
};

// Thread-partial real-space energy of one site against the framework (voxel list) and the
// guest sites outside [ex_lo, ex_hi).  Threads stride by `nthr` starting at `tid`.
__device__ __forceinline__ void site_partial(const DevSystem& S, const GuestView& G, const PendingCommit& P, double px,
                                             double py, double pz, double q, int ty, int ex_lo, int ex_hi, int tid,
                                             int nthr, double& ec_fw, double& ev_fw, double& ec_g, double& ev_g) {
  const double chgea = q * kR4pie0;
  const int* prow = S.pair_row + ty * (S.ntypes + 1);
  for (int sg = 0; sg < G.nseg; sg++) {
    int lo = G.seg_off[sg], hi = lo + G.seg_len[sg];
    for (int j = lo + tid; j < hi; j += nthr) {
      if (j >= ex_lo && j < ex_hi) continue;
      double4 a;
      int t;
      if (sg != P.seg || j < P.lo) {
        a = G.site[j];
        t = G.type[j];
      } else if (P.op == kDelete) {  // the sites after the removed molecule, one molecule on
        a = G.site[j + P.ns];
        t = G.type[j + P.ns];
      } else if (j < P.lo + P.ns) {  // the inserted or displaced molecule
        a = P.site[j - P.lo];
        t = P.type[j - P.lo];
      } else {
        a = G.site[j];
        t = G.type[j];
      }
      pair_energy(S, px - a.x, py - a.y, pz - a.z, chgea, a.w, prow[t], ec_g, ev_g);
    }
  }
  int v = voxel_of(S, px, py, pz);
  int b = S.vox_off[v], e = S.vox_off[v + 1];
  for (int i = b + tid; i < e; i += nthr) {
    double4 a = S.vox_xyzq[i];
    pair_energy(S, px - a.x, py - a.y, pz - a.z, chgea, a.w, prow[S.vox_type[i]], ec_fw, ev_fw);
  }
}

// Deterministic block sum of NV values per thread (fixed shuffle tree + fixed warp order).
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double* red /* >= 32*NV */) {
#pragma unroll
  for (int k = 0; k < NV; k++)
    for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
  int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  __syncthreads();
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < NV; k++) red[w * NV + k] = v[k];
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < NV; k++) {
      double s = 0.0;
      for (int i = 0; i < nw; i++) s += red[i * NV + k];
      v[k] = s;
    }
  }
}

#endif  // __CUDACC__

}  // namespace fmc
