// Persistent batched kernel: one CTA (256 threads) per chain runs `moves` iterations of the
// move loop (gcmc.f:589-1380) entirely on the device.
//
// Per move: thread 0 draws the random numbers, picks and builds the trial (duni, move choice,
// step-size adaptation, random_ins / random_disp), all threads then build the trial sites'
// phase tables in shared memory, sweep their k-vectors (S(k), S_new, akk and the k-vector table
// are resident in shared memory for the whole launch) and their share of the real-space pair
// candidates (framework voxel list + guest sites), one fixed-order block reduction gives
// {sum akk*d|S|^2, ewld2, vdw}, thread 0 applies energy_eval, and on acceptance every thread
// commits its own k-vectors while the block updates the guest-site segment.
#include <cstring>

#include "fmc_batch.h"

namespace fmc {

namespace {

struct MoveSmem {
  int mtype, g, mol, nold, nnew, accepted, ex_lo, ex_hi;
  int commit_lo, seg_end, ns, randchoice, need_lrc;
  double delrc, rande;
  double x[2 * kBatchMaxSites], y[2 * kBatchMaxSites], z[2 * kBatchMaxSites], q[2 * kBatchMaxSites];
  int type[2 * kBatchMaxSites];
  // real-space work list: per trial site its voxel-list start/length and the prefix of
  // candidates (voxel entries + every guest site) over the sites
  int vb[2 * kBatchMaxSites], vl[2 * kBatchMaxSites], pre[2 * kBatchMaxSites + 1];
  int gpre[kMaxGuestTypes + 1];
  double lrc_term[kBatchMaxTab];
};

__device__ double lrc_device(const SysConst& Y, const int* numtyp) {
  if (!Y.lrc_on) return 0.0;
  const double twopi = 2.0 * kPi, v = Y.volm;
  double e = 0.0;
  int ivdw = 0;
  for (int i = 1; i <= Y.ntypes; i++)
    for (int j = 1; j <= i; j++) {
      ivdw++;
      double den =
          twopi * ((double)numtyp[i] * (double)numtyp[j] - (double)Y.numfrz[i] * (double)Y.numfrz[j]) / (v * v);
      e = e + v * den * Y.steadd[ivdw];
    }
  return e;
}

// Thread 0: bookkeeping of gcmc.f:594-736 (production / termination every 400 moves),
// random choices and the trial sites.
__device__ __noinline__ void move_begin(ChainDev& C, const SysConst& Y, const DevSystem& S, MoveSmem& M) {
  C.prof[7] -= clock64();
  C.gcmccount++;
  if (C.gcmccount % 400 == 0) {
    int totalguests = 0;
    for (int g = 0; g < Y.nspecies; g++) totalguests += C.nmol[g];
    if (C.production) {
      if (C.mcsteps < 0) {
        for (int t = 4; t > 0; t--) C.tick[t] = C.tick[t - 1];
        C.tick[0] = !(C.prodcount < (long long)(-C.mcsteps) * (totalguests + 1));
        bool all = true;
        for (int t = 0; t < 5; t++) all = all && C.tick[t];
        if (all) C.lgchk = 0;
      } else if (C.prodcount >= C.mcsteps) {
        C.lgchk = 0;
      }
    } else if (C.eqsteps > 0) {
      if (C.gcmccount >= C.eqsteps) C.production = 1;
    } else if (C.eqsteps < 0) {
      for (int t = 4; t > 0; t--) C.tick[t] = C.tick[t - 1];
      C.tick[0] = !((long long)C.gcmccount < (long long)(-C.eqsteps) * (totalguests + 1));
      bool all = true;
      for (int t = 0; t < 5; t++) all = all && C.tick[t];
      if (all) {
        C.production = 1;
        for (int t = 0; t < 5; t++) C.tick[t] = 0;
      }
    }
  }
  const int ng = Y.nspecies;
  int g = 0;
  if (ng > 1) g = (int)floor(duni_next(C.rng) * ng);
  double randmov = duni_next(C.rng);
  const double* c = C.mvcum[g];
  int mtype;
  if (randmov < c[0]) mtype = kInsert;
  else if (randmov < c[1]) mtype = kDelete;
  else if (randmov < c[2]) mtype = kDisplace;
  else if (randmov < c[5]) mtype = -1;
  else if (randmov < c[6]) mtype = kTranslate;
  else if (randmov < c[7]) mtype = kRotate;
  else if (randmov < c[8]) mtype = -1;
  else mtype = kDisplace;
  const SpeciesConst& P = Y.sp[g];
  const int ns = P.nsite, nmols = C.nmol[g];
  // step-size adaptation (gcmc.f:794-834)
  if (nmols >= 1 && C.disp_count[g] >= 1) {
    if (C.disp_count[g] % 100 == 0) {
      if ((C.accept_disp[g] / (double)C.disp_count[g]) > C.disp_ratio[g]) C.delrdisp[g] = C.delrdisp[g] * 1.05;
      else if (C.delrdisp[g] > kDelrMin) C.delrdisp[g] = C.delrdisp[g] * 0.95;
    } else if (C.disp_count[g] % 50 == 0) {
      if ((C.accept_disp[g] / (double)C.disp_count[g]) > C.disp_ratio[g]) C.rotangle = C.rotangle * 1.05;
      else if (C.rotangle > kMinAngle) C.rotangle = C.rotangle * 0.95;
    }
  }
  if (nmols >= 1 && C.tran_count[g] >= 1 && C.tran_count[g] % 100 == 0) {
    if ((C.accept_tran[g] / (double)C.tran_count[g]) > C.tran_ratio[g]) C.tran_delr[g] = C.tran_delr[g] * 1.05;
    else if (C.tran_delr[g] > kDelrMin) C.tran_delr[g] = C.tran_delr[g] * 0.95;
  }
  if (nmols >= 1 && C.rota_count >= 1 && C.rota_count % 100 == 0) {
    if ((C.accept_rota / (double)C.rota_count) > C.rota_ratio) C.rota_rotangle = C.rota_rotangle * 1.05;
    else if (C.rota_rotangle > kMinAngle) C.rota_rotangle = C.rota_rotangle * 0.95;
  }
  if (nmols == 0) mtype = kInsert;
  C.prof[7] += clock64();  // minus the stamp taken at entry: selection + adaptation
  M.mtype = mtype;
  M.g = g;
  M.ns = ns;
  M.mol = -1;
  M.randchoice = 0;
  M.ex_lo = M.ex_hi = -1;
  M.nold = M.nnew = 0;
  M.delrc = 0.0;
  M.rande = -1.0;
  M.need_lrc = 0;
  if (mtype < 0) {
    C.status = 3;
    return;
  }
  double* x = M.x;
  double* y = M.y;
  double* z = M.z;
  C.prof[8] -= clock64();  // trial generation and site loads
  if (mtype == kInsert) {
    C.ins_count++;
    if ((C.totatm - C.framatm) + ns >= C.maxguest || (nmols + 1) * ns > C.seg_cap[g]) {
      C.status = 75;
      return;
    }
    double r[7];
    for (int i = 0; i < 7; i++) r[i] = duni_next(C.rng);
    trial_insert(S.cell, P.tx, P.ty, P.tz, ns, r, x, y, z);
    M.nnew = ns;
    for (int i = 0; i < ns; i++) C.numtyp[P.type[i]]++;
    M.need_lrc = 1;
  } else if (mtype == kDelete) {
    C.del_count++;
    int randchoice = (int)floor(duni_next(C.rng) * nmols) + 1;
    M.randchoice = randchoice;
    M.mol = randchoice - 1;
    M.ex_lo = C.seg_off[g] + M.mol * ns;
    M.ex_hi = M.ex_lo + ns;
    for (int i = 0; i < ns; i++) {
      double4 a = C.gsite[M.ex_lo + i];
      x[i] = a.x;
      y[i] = a.y;
      z[i] = a.z;
    }
    M.nold = ns;
    for (int i = 0; i < ns; i++) C.numtyp[P.type[i]]--;
    M.need_lrc = 1;
  } else {
    double r[7], dis_delr, dis_rot;
    if (mtype == kTranslate) {
      C.tran_count[g]++;
      r[0] = duni_next(C.rng);
      r[1] = duni_next(C.rng);
      r[2] = duni_next(C.rng);
      r[3] = r[4] = r[5] = r[6] = 0.0;
      dis_delr = C.tran_delr[g];
      dis_rot = 0.0;
    } else if (mtype == kRotate) {
      C.rota_count++;
      r[0] = r[1] = r[2] = 0.5;
      for (int i = 3; i < 7; i++) r[i] = duni_next(C.rng);
      dis_delr = 0.0;
      dis_rot = C.rota_rotangle;
    } else {
      C.disp_count[g]++;
      for (int i = 0; i < 7; i++) r[i] = duni_next(C.rng);
      dis_delr = C.delrdisp[g];
      dis_rot = C.rotangle;
    }
    int randchoice = (int)floor(duni_next(C.rng) * nmols) + 1;
    M.randchoice = randchoice;
    M.mol = randchoice - 1;
    M.ex_lo = C.seg_off[g] + M.mol * ns;
    M.ex_hi = M.ex_lo + ns;
    for (int i = 0; i < ns; i++) {
      double4 a = C.gsite[M.ex_lo + i];
      x[i] = a.x;
      y[i] = a.y;
      z[i] = a.z;
      x[ns + i] = a.x;
      y[ns + i] = a.y;
      z[ns + i] = a.z;
    }
    trial_displace(S.cell, P.mass, ns, dis_delr, dis_rot, r, x + ns, y + ns, z + ns);
    M.nold = ns;
    M.nnew = ns;
  }
  for (int i = 0; i < M.nold + M.nnew; i++) {
    int s = i < M.nold ? i : i - M.nold;
    M.q[i] = P.q[s];
    M.type[i] = P.type[s];
  }
  C.prof[8] += clock64();
}

// Thread 0: energy assembly, energy_eval, counters, statistics (gcmc.f:941-1380, 1814-1860).
__device__ __noinline__ void move_end(ChainDev& C, const SysConst& Y, MoveSmem& M, const double v[3], MoveRecord* rec) {
  const int g = M.g, ns = M.ns, mtype = M.mtype;
  const SpeciesConst& P = Y.sp[g];
  const int nmols = C.nmol[g];
  double ewld1 = Y.S.recip_pref * v[0];
  double ewld3 = 0.0, estep;
  bool accepted;
  if (mtype == kInsert) {
    ewld1 = ewld1 + P.engsic;
    ewld3 = P.ewald3en;
    estep = (ewld1 + v[1] + ewld3 + v[2] + M.delrc) / Y.engunit;
    M.rande = duni_next(C.rng);
    accepted = accept_move(estep, M.rande, Y.statvolm, C.press[g], nmols, C.temp, C.beta, kInsert);
  } else if (mtype == kDelete) {
    ewld1 = ewld1 - P.engsic;
    ewld3 = P.ewald3en;
    estep = (ewld1 - v[1] - ewld3 - v[2] + M.delrc) / Y.engunit;
    M.rande = duni_next(C.rng);
    accepted = accept_move(estep, M.rande, Y.statvolm, C.press[g], nmols, C.temp, C.beta, kDelete);
  } else {
    estep = (ewld1 + v[1] + v[2]) / Y.engunit;
    if (estep < 0.0) {
      accepted = true;
    } else {
      M.rande = duni_next(C.rng);
      accepted = accept_move(estep, M.rande, Y.statvolm, C.press[g], nmols, C.temp, C.beta, kDisplace);
    }
  }
  M.accepted = accepted;
  M.seg_end = C.seg_off[g] + nmols * ns;
  if (mtype == kInsert) {
    M.commit_lo = M.seg_end;
    if (accepted) {
      C.accept_ins++;
      C.elrc = C.elrc + M.delrc;
      C.nmol[g]++;
      C.totatm += ns;
      C.energy[g] += estep;
    } else {
      for (int i = 0; i < ns; i++) C.numtyp[P.type[i]]--;
    }
  } else if (mtype == kDelete) {
    M.commit_lo = M.ex_lo;
    if (accepted) {
      C.accept_del++;
      C.elrc = C.elrc + M.delrc;
      C.nmol[g]--;
      C.totatm -= ns;
      C.energy[g] += estep;
    } else {
      for (int i = 0; i < ns; i++) C.numtyp[P.type[i]]++;
    }
  } else {
    M.commit_lo = M.ex_lo;
    if (accepted) {
      if (mtype == kTranslate) C.accept_tran[g]++;
      else if (mtype == kRotate) C.accept_rota++;
      else C.accept_disp[g]++;
      C.energy[g] += estep;
    }
  }
  if (C.production && ((C.laccsample && accepted) || !C.laccsample)) {
    C.prodcount++;
    double pc = (double)C.prodcount;
    for (int i = 0; i < Y.nspecies; i++) {
      double dm = (double)C.nmol[i], m2 = dm * dm, en = C.energy[i], e2 = en * en;
      double* cs = C.stats[i];
      cs[0] = cs[0] + (dm - cs[0]) / pc;
      cs[1] = cs[1] + (en - cs[1]) / pc;
      cs[2] = cs[2] + (en * dm - cs[2]) / pc;
      cs[3] = cs[3] + (m2 - cs[3]) / pc;
      cs[4] = cs[4] + (e2 - cs[4]) / pc;
    }
  }
  C.moves_done++;
  if (rec) {
    rec->step = C.gcmccount;
    rec->iguest = g;
    rec->mtype = mtype;
    rec->randchoice = M.randchoice;
    rec->accepted = accepted;
    rec->nmols_after = C.nmol[g];
    rec->pad0 = rec->pad1 = 0;
    rec->ewld1 = ewld1;
    rec->ewld2 = v[1];
    rec->ewld3 = ewld3;
    rec->vdw = v[2];
    rec->delrc = M.delrc;
    rec->estep = estep;
    rec->rande = M.rande;
    rec->energy_after = C.energy[g];
  }
}

// Tail correction (gstlrcorrect, vdw_terms.f:684-745) by one warp: lane-parallel pair terms,
// summed by lane 0 in the reference's pair order.
__device__ __forceinline__ void lrc_warp(const ChainDev& C, const SysConst& Y, MoveSmem& M, int lane) {
  const int nt = Y.ntypes, ntab = nt * (nt + 1) / 2;
  const double twopi = 2.0 * kPi, v = Y.volm;
  for (int p = lane; p < ntab; p += 32) {
    int i = 1;
    while (i * (i + 1) / 2 <= p) i++;
    int j = p - (i - 1) * i / 2 + 1;
    double den =
        twopi * ((double)C.numtyp[i] * (double)C.numtyp[j] - (double)Y.numfrz[i] * (double)Y.numfrz[j]) / (v * v);
    M.lrc_term[p] = v * den * Y.steadd[p + 1];
  }
  __syncwarp();
  if (lane == 0) {
    double e = 0.0;
    if (Y.lrc_on)
      for (int p = 0; p < ntab; p++) e = e + M.lrc_term[p];
    M.delrc = e - C.elrc;
  }
}

// One real-space candidate: a framework atom from a site's voxel list or a guest site.
struct Cand {
  double4 a;
  int type, site;
  bool live;
};

__device__ __forceinline__ Cand fetch_candidate(const DevSystem& S, const ChainDev& C, const MoveSmem& M, int nseg,
                                                int t, int& s) {
  Cand c;
  c.live = false;
  c.site = s;
  if (t >= M.pre[M.nold + M.nnew]) return c;
  while (t >= M.pre[s + 1]) s++;
  c.site = s;
  int j = t - M.pre[s];
  if (j < M.vl[s]) {
    c.a = S.vox_xyzq[M.vb[s] + j];
    c.type = S.vox_type[M.vb[s] + j];
    c.live = true;
  } else {
    int jg = j - M.vl[s], g = 0;
    while (g + 1 < nseg && jg >= M.gpre[g + 1]) g++;
    int site_idx = C.seg_off[g] + (jg - M.gpre[g]);
    if (site_idx < M.ex_lo || site_idx >= M.ex_hi) {
      c.a = C.gsite[site_idx];
      c.type = C.gtype[site_idx];
      c.live = true;
    }
  }
  return c;
}

__global__ void __launch_bounds__(kBatchThreads, 2) fmc_batch_kernel(BatchLaunch L, int tab_stride) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ ChainDev C;
  __shared__ MoveSmem M;
  __shared__ SysConst Ysm;
  __shared__ double red[32 * 3];
  __shared__ int prow_s[(kBatchMaxTypes + 1) * (kBatchMaxTypes + 1)];
  DevSystem& S = Ysm.S;
  const int tid = threadIdx.x, cidx = blockIdx.x, warp = tid >> 5, lane = tid & 31;
  if (cidx >= L.nchains) return;
  {
    const int* src = reinterpret_cast<const int*>(&L.chains[cidx]);
    int* dst = reinterpret_cast<int*>(&C);
    for (int i = tid; i < (int)(sizeof(ChainDev) / sizeof(int)); i += blockDim.x) dst[i] = src[i];
  }
  __syncthreads();
  {
    const int* src = reinterpret_cast<const int*>(&L.systems[C.sys]);
    int* dst = reinterpret_cast<int*>(&Ysm);
    for (int i = tid; i < (int)(sizeof(SysConst) / sizeof(int)); i += blockDim.x) dst[i] = src[i];
  }
  __syncthreads();
  const SysConst& Y = Ysm;
  const int K = S.K, Kmax = L.kmax_smem, nseg = Y.nspecies;
  const int nt1 = S.ntypes + 1;
  for (int i = tid; i < nt1 * nt1; i += blockDim.x) prow_s[i] = S.pair_row[i];
  double2* Sk = reinterpret_cast<double2*>(smem_raw);
  double2* Sn = Sk + Kmax;
  double* ak = reinterpret_cast<double*>(Sn + Kmax);
  int* kp = reinterpret_cast<int*>(ak + Kmax);
  double2* tab = reinterpret_cast<double2*>(kp + ((Kmax + 3) & ~3));
  for (int k = tid; k < K; k += blockDim.x) {
    Sk[k] = C.sk[k];
    ak[k] = S.akk[k];
    kp[k] = S.kpack[k];
  }
  const int k1 = S.kmax[0], k2 = S.kmax[1], k3 = S.kmax[2];
  const int stride = k1 + k2 + k3 + 3;
  (void)tab_stride;
  __syncthreads();
  long long t0 = 0, t1 = 0;
  const bool prof = L.profile != 0;
  for (int mv = 0; mv < L.moves; mv++) {
    if (prof && tid == 0) t0 = clock64();
    if (tid == 0) move_begin(C, Y, S, M);
    __syncthreads();
    if (prof && tid == 0) {
      t1 = clock64();
      C.prof[0] += t1 - t0;
      t0 = t1;
    }
    if (C.status) break;
    const int nsite = M.nold + M.nnew;
    if (warp == 0) {
      // phase tables of the trial sites (ewald.f:95-137)
      for (int w = lane; w < nsite * 3; w += 32) {
        int st = w / 3, ax = w % 3;
        double f[3];
        frac_coords(S.cell, M.x[st], M.y[st], M.z[st], f);
        axis_phases(f[ax], S.kmax[ax], tab + st * stride + (ax == 0 ? 0 : (ax == 1 ? k1 + 1 : k1 + k2 + 2)));
      }
    } else if (warp == 1) {
      if (M.need_lrc) lrc_warp(C, Y, M, lane);
    } else if (warp == 2) {
      // real-space work list: voxel list of every trial site, then every guest site
      if (lane < nsite) {
        int v = voxel_of(S, M.x[lane], M.y[lane], M.z[lane]);
        M.vb[lane] = S.vox_off[v];
        M.vl[lane] = S.vox_off[v + 1] - S.vox_off[v];
      }
      __syncwarp();
      if (lane == 0) {
        int gt = 0;
        M.gpre[0] = 0;
        for (int g = 0; g < nseg; g++) {
          gt += C.nmol[g] * Y.sp[g].nsite;
          M.gpre[g + 1] = gt;
        }
        M.pre[0] = 0;
        for (int st = 0; st < nsite; st++) M.pre[st + 1] = M.pre[st] + M.vl[st] + gt;
      }
    }
    __syncthreads();
    if (prof && tid == 0) {
      t1 = clock64();
      C.prof[1] += t1 - t0;
      t0 = t1;
    }
    double v[3] = {0.0, 0.0, 0.0};
    const int mtype = M.mtype, nold = M.nold;
    // ---- reciprocal space: this thread's k-vectors
    for (int k = tid; k < K; k += blockDim.x) {
      int l, m, n;
      kunpack(kp[k], l, m, n);
      int am = m < 0 ? -m : m, an = n < 0 ? -n : n;
      double2 aold = make_double2(0.0, 0.0), anew = make_double2(0.0, 0.0);
      for (int st = 0; st < nsite; st++) {
        const double2* t = tab + st * stride;
        double2 c = m >= 0 ? cmul(t[l], t[k1 + 1 + am]) : cmulc(t[l], t[k1 + 1 + am]);
        c = n >= 0 ? cmul(c, t[k1 + k2 + 2 + an]) : cmulc(c, t[k1 + k2 + 2 + an]);
        double q = M.q[st];
        if (st < nold) {
          aold.x += q * c.x;
          aold.y += q * c.y;
        } else {
          anew.x += q * c.x;
          anew.y += q * c.y;
        }
      }
      double2 so = Sk[k], sn;
      if (mtype == kInsert)
        sn = make_double2(anew.x + so.x, anew.y + so.y);
      else if (mtype == kDelete)
        sn = make_double2(so.x - aold.x, so.y - aold.y);
      else
        sn = make_double2((so.x - aold.x) + anew.x, (so.y - aold.y) + anew.y);
      Sn[k] = sn;
      v[0] += ak[k] * (sn.x * sn.x + sn.y * sn.y - so.x * so.x - so.y * so.y);
    }
    if (prof && tid == 0) C.prof[5] += clock64() - t0;
    // ---- real space: every (site, candidate) pair, four candidates in flight per thread
    {
      const bool sub_old = (mtype != kInsert && mtype != kDelete);
      const int T = M.pre[nsite];
      int s0 = 0, s1 = 0, s2 = 0, s3 = 0;
      for (int base = tid; base < T; base += 4 * kBatchThreads) {
        Cand c[4];
        c[0] = fetch_candidate(S, C, M, nseg, base, s0);
        c[1] = fetch_candidate(S, C, M, nseg, base + kBatchThreads, s1);
        c[2] = fetch_candidate(S, C, M, nseg, base + 2 * kBatchThreads, s2);
        c[3] = fetch_candidate(S, C, M, nseg, base + 3 * kBatchThreads, s3);
#pragma unroll
        for (int u = 0; u < 4; u++) {
          if (!c[u].live) continue;
          const int st = c[u].site;
          double ec = 0.0, ev = 0.0;
          pair_energy(S, M.x[st] - c[u].a.x, M.y[st] - c[u].a.y, M.z[st] - c[u].a.z, M.q[st] * kR4pie0, c[u].a.w,
                      prow_s[M.type[st] * nt1 + c[u].type], ec, ev);
          if (sub_old && st < nold) {
            v[1] -= ec;
            v[2] -= ev;
          } else {
            v[1] += ec;
            v[2] += ev;
          }
        }
      }
    }
    if (prof && tid == 0) C.prof[6] += clock64() - t0;
    block_sum<3>(v, red);
    if (prof && tid == 0) {
      t1 = clock64();
      C.prof[2] += t1 - t0;
      t0 = t1;
    }
    if (tid == 0) move_end(C, Y, M, v, L.trace ? L.trace + (size_t)cidx * L.moves + mv : nullptr);
    __syncthreads();
    if (prof && tid == 0) {
      t1 = clock64();
      C.prof[3] += t1 - t0;
      t0 = t1;
    }
    if (M.accepted) {
      for (int k = tid; k < K; k += blockDim.x) Sk[k] = Sn[k];
      const int ns = M.ns;
      if (mtype == kDelete) {
        const int lo = M.commit_lo, end = M.seg_end;
        for (int base = lo; base < end - ns; base += blockDim.x) {
          int i = base + tid;
          bool act = i < end - ns;
          double4 a = make_double4(0, 0, 0, 0);
          int t = 0;
          if (act) {
            a = C.gsite[i + ns];
            t = C.gtype[i + ns];
          }
          __syncthreads();
          if (act) {
            C.gsite[i] = a;
            C.gtype[i] = t;
          }
          __syncthreads();
        }
      } else if (tid < ns) {
        int st = (mtype == kInsert) ? tid : ns + tid;
        C.gsite[M.commit_lo + tid] = make_double4(M.x[st], M.y[st], M.z[st], M.q[st]);
        C.gtype[M.commit_lo + tid] = M.type[st];
      }
    }
    __syncthreads();
    if (prof && tid == 0) C.prof[4] += clock64() - t0;
  }
  for (int k = tid; k < K; k += blockDim.x) C.sk[k] = Sk[k];
  __syncthreads();
  {
    const int* src = reinterpret_cast<const int*>(&C);
    int* dst = reinterpret_cast<int*>(&L.chains[cidx]);
    for (int i = tid; i < (int)(sizeof(ChainDev) / sizeof(int)); i += blockDim.x) dst[i] = src[i];
  }
}

}  // namespace

int batch_smem_bytes(int kmax_K, int tab_sites, int tab_stride) {
  return kmax_K * (int)(2 * sizeof(double2) + sizeof(double)) + ((kmax_K + 3) & ~3) * (int)sizeof(int) +
         tab_sites * tab_stride * (int)sizeof(double2);
}

cudaError_t configure_batch_kernel(int smem_bytes) {
  return cudaFuncSetAttribute(fmc_batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_bytes);
}

cudaError_t launch_batch(const BatchLaunch& L, int smem_bytes, int tab_stride, cudaStream_t st) {
  fmc_batch_kernel<<<L.nchains, kBatchThreads, smem_bytes, st>>>(L, tab_stride);
  return cudaGetLastError();
}

}  // namespace fmc
