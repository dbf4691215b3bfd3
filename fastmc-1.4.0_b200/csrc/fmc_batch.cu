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
#include <map>
#include <mutex>

#include "fmc_batch.h"

namespace fmc {

namespace {

struct MoveSmem {
  int mtype, g, mol, nold, nnew, accepted, ex_lo, ex_hi;
  int commit_lo, seg_end, ns, randchoice, need_lrc, rande_drawn;
  double delrc, rande;
  double r[7], dis_delr, dis_rot;  // the trial's random numbers and step sizes (select_move)
  double ewld1, ewld2, vdw, ewld3, estep;
  double x[2 * kBatchMaxSites], y[2 * kBatchMaxSites], z[2 * kBatchMaxSites], q[2 * kBatchMaxSites];
  int type[2 * kBatchMaxSites];
  // real-space work list: per trial site its voxel-list start/length and the prefix of
  // candidates (voxel entries + every guest site) over the sites
  int vb[2 * kBatchMaxSites], vl[2 * kBatchMaxSites], pre[2 * kBatchMaxSites + 1];
  int gpre[kMaxGuestTypes + 1];
  double lrc_term[kBatchMaxTab];
  // multi-jump (gcmc.f:1557-1785) across the two loop trips of one move: stage 1 while the
  // first jump is evaluated and committed, 2 for the second jump; the first molecule's choice
  // and old sites, its energy change, the energy before the move and the commit action
  // (1: park S(k) in the chain's global copy, then commit; 2: restore S(k) and the first molecule)
  int mj_stage, mj_first, mj_lo, mj_action;
  double mj_estep, mj_energy0;
  double mj_old[3 * kBatchMaxSites];
};

// duni (gcmc.f:2712-2805) with ir, jr and c held in registers across a run of draws; the
// arithmetic is duni_next's, draw for draw.
struct DuniLocal {
  float* u;
  float c;
  int ir, jr;
  __device__ explicit DuniLocal(Duni& d) : u(d.u), c(d.c), ir(d.ir), jr(d.jr) {}
  __device__ void store(Duni& d) const {
    d.c = c;
    d.ir = ir;
    d.jr = jr;
  }
  __device__ double next() {
    const float cd = 7654321.0f / 16777216.0f, cm = 16777213.0f / 16777216.0f;
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

// Thread 0: bookkeeping of gcmc.f:594-736 (production / termination every 400 moves),
// random choices and the trial sites.
// Thread 0, every 400 moves (gcmc.f:594-736): the end of production, the switch to production
// and the pressure equilibration; a rare path, kept out of line.
__device__ __noinline__ void check400(ChainDev& C, const SysConst& Y) {
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
  } else {
    if (C.despre > 0) {  // pressure equilibration (gcmc.f:637-696)
      for (int t = 4; t > 0; t--) C.tick[t] = C.tick[t - 1];
      C.tick[0] = !(C.prodcount < (long long)(-C.eqsteps) * (totalguests + 1) / 4);
      if (C.tick[0])
        pressure_adjust(Y.nspecies, C.press, &C.stats[0][0], 6, C.adspres, C.adsguen, C.packf, Y.volm, C.temp,
                        C.presrate, C.despre, C.gcmccount, C.prodcount, C.eqsteps);
    }
    if (C.eqsteps > 0) {
      if (C.gcmccount >= C.eqsteps && C.despre == 0) C.production = 1;
    } else if (C.eqsteps < 0) {
      for (int t = 4; t > 0; t--) C.tick[t] = C.tick[t - 1];
      C.tick[0] = !((long long)C.gcmccount < (long long)(-C.eqsteps) * (totalguests + 1));
      if (C.despre > 0) C.tick[0] = 0;
      bool all = true;
      for (int t = 0; t < 5; t++) all = all && C.tick[t];
      if (all) {
        C.production = 1;
        for (int t = 0; t < 5; t++) C.tick[t] = 0;
      }
    }
  }
}

// Thread 0: energy assembly of the move (gcmc.f:946, 1112, 1328).  v = {sum akk*d|S|^2,
// ewld2, vdw} as reduced by the block.
__device__ __forceinline__ void assemble(const SysConst& Y, MoveSmem& M, const double* v) {
  const SpeciesConst& P = Y.sp[M.g];
  M.ewld1 = Y.S.recip_pref * v[0];
  M.ewld2 = v[1];
  M.vdw = v[2];
  M.ewld3 = 0.0;
  if (M.mtype == kInsert) {
    M.ewld1 = M.ewld1 + P.engsic;
    M.ewld3 = P.ewald3en;
    M.estep = (M.ewld1 + v[1] + M.ewld3 + v[2] + M.delrc) / Y.engunit;
  } else if (M.mtype == kDelete) {
    M.ewld1 = M.ewld1 - P.engsic;
    M.ewld3 = P.ewald3en;
    M.estep = (M.ewld1 - v[1] - M.ewld3 - v[2] + M.delrc) / Y.engunit;
  } else {
    M.estep = (M.ewld1 + v[1] + v[2]) / Y.engunit;
  }
}

// Thread 0: acceptance (energy_eval, utility_pack.f:3049-3095, with the displacement
// shortcut of gcmc.f:1330-1338).  Random numbers are drawn exactly where the reference draws them.
__device__ __forceinline__ void decide(ChainDev& C, const SysConst& Y, MoveSmem& M) {
  const int g = M.g, mtype = M.mtype, nmols = C.nmol[g];
  double e = M.estep;
  if (mtype == kNoop) {  // nothing to accept or reject; no draw
    M.accepted = 0;
    return;
  }
  if (mtype == kMultiJump) {
    if (M.mj_stage == 1) {  // the first jump is kept for now
      M.accepted = 1;
      return;
    }
    e = M.mj_estep + e;  // one test on the summed change (gcmc.f:1730-1739)
  }
  if (mtype == kInsert || mtype == kDelete) {
    M.rande = duni_next(C.rng);
    M.rande_drawn = 1;
    M.accepted = accept_move(e, M.rande, Y.statvolm, C.press[g], nmols, C.temp, C.beta, mtype);
    return;
  }
  if (e < 0.0) {
    M.accepted = 1;
    return;
  }
  M.rande = duni_next(C.rng);
  M.rande_drawn = 1;
  M.accepted = accept_move(e, M.rande, Y.statvolm, C.press[g], nmols, C.temp, C.beta, kDisplace);
}

// Thread 0: counters, running energy, statistics and the trace record (gcmc.f:954-1380,
// 1814-1860) once the move is decided.
// Thread 0, production moves: the rolling averages, the stored samples and the averaging
// windows of gcmc.f:1814-1928.  ins_g: species of an accepted insertion (-1: none).
__device__ __noinline__ void production_sample(ChainDev& C, const SysConst& Y, int ins_g, bool counted,
                                               double estep) {
  if ((C.laccsample && counted) || !C.laccsample) {
    C.prodcount++;
    C.win.rollcount++;
    const double pc = (double)C.prodcount;
    for (int i = 0; i < Y.nspecies; i++) {
      double dm = (double)(float)C.nmol[i], m2 = dm * dm, en = C.energy[i], e2 = en * en;
      if (C.gasmol && C.prodcount <= kSampleCap + 1) {
        C.gasmol[(size_t)i * kSampleCap + C.prodcount - 1] = dm;
        C.gaseng[(size_t)i * kSampleCap + C.prodcount - 1] = en;
      }
      double* cs = C.stats[i];
      cs[0] = cs[0] + (dm - cs[0]) / pc;
      cs[1] = cs[1] + (en - cs[1]) / pc;
      cs[2] = cs[2] + (en * dm - cs[2]) / pc;
      cs[3] = cs[3] + (m2 - cs[3]) / pc;
      cs[4] = cs[4] + (e2 - cs[4]) / pc;
      window_sample(C.win, i, dm, en, ins_g == i, estep, C.temp, C.accept_ins, cs);
    }
  }
  if (C.prodcount % C.nwind == 0 || !C.lgchk)
    window_close(C.win, Y.nspecies, C.nwind, C.temp, [&C](int i) { return (const double*)C.stats[i]; });
}

__device__ __noinline__ void bookkeep(ChainDev& C, const SysConst& Y, MoveSmem& M, MoveRecord* rec) {
  const int g = M.g, ns = M.ns, mtype = M.mtype;
  const SpeciesConst& P = Y.sp[g];
  const int nmols = C.nmol[g];
  const bool accepted = M.accepted;
  double estep = M.estep;
  M.seg_end = C.seg_off[g] + nmols * ns;
  if (mtype == kMultiJump) {
    M.commit_lo = M.ex_lo;
    if (M.mj_stage == 1) {
      // the first jump stands while the second is tried (gcmc.f:1697-1715): remember where it
      // came from; the move is counted once, when the second jump is decided
      M.mj_estep = estep;
      M.mj_lo = M.ex_lo;
      for (int i = 0; i < ns; i++) {
        M.mj_old[3 * i] = M.x[i];
        M.mj_old[3 * i + 1] = M.y[i];
        M.mj_old[3 * i + 2] = M.z[i];
      }
      M.mj_action = 1;
      C.energy[g] = M.mj_energy0 + estep;
      return;
    }
    estep = M.mj_estep + estep;
    M.mj_stage = 0;
    if (accepted) {
      C.accept_jump++;
      C.energy[g] = M.mj_energy0 + estep;
    } else {
      M.mj_action = 2;
      C.energy[g] = M.mj_energy0;
    }
  }
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
  } else if (mtype != kNoop && mtype != kMultiJump) {
    M.commit_lo = M.ex_lo;
    if (accepted) {
      if (mtype == kTranslate) C.accept_tran[g]++;
      else if (mtype == kRotate) C.accept_rota++;
      else if (mtype == kJump) C.accept_jump++;
      else C.accept_disp[g]++;
      C.energy[g] += estep;
    }
  }
  // flex / swap leave the reference's `accepted` as the previous move set it
  const bool counted = mtype == kNoop ? (C.last_accepted != 0) : accepted;
  if (mtype != kNoop) C.last_accepted = accepted;
  if (C.production) production_sample(C, Y, mtype == kInsert && accepted ? g : -1, counted, estep);
  else if (C.despre > 0 && ((C.laccsample && counted) || !C.laccsample)) {
    // running loading while the pressures equilibrate (gcmc.f:1796-1808)
    C.prodcount++;
    for (int i = 0; i < Y.nspecies; i++)
      C.stats[i][0] = C.stats[i][0] + ((double)(float)C.nmol[i] - C.stats[i][0]) / (double)C.prodcount;
  }
  C.last_dE = accepted ? estep : 0.0;
  C.moves_done++;
  if (rec) {
    rec->step = C.gcmccount;
    rec->iguest = g;
    rec->mtype = mtype;
    rec->randchoice = M.randchoice;
    rec->accepted = counted;  // as the reference's `accepted` reads after the move
    rec->nmols_after = C.nmol[g];
    rec->pad0 = 0;
    rec->pad1 = 0;
    rec->ewld1 = M.ewld1;
    rec->ewld2 = M.ewld2;
    rec->ewld3 = M.ewld3;
    rec->vdw = M.vdw;
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

// Device clock in nanoseconds (%globaltimer: one time base for every SM, unlike clock64).
__device__ __forceinline__ long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return (long long)t;
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
    const int site_idx = C.seg_off[g] + (jg - M.gpre[g]);
    if (site_idx < M.ex_lo || site_idx >= M.ex_hi) {
      c.a = C.gsite[site_idx];
      c.type = C.gtype[site_idx];
      c.live = true;
    }
  }
  return c;
}

// Warp 0: phase tables of the trial sites (ewald.f:95-137).
__device__ __forceinline__ void build_phases(const DevSystem& S, const MoveSmem& M, void* tabv, int stride, int lane) {
  const int nsite = M.nold + M.nnew, k1 = S.kmax[0], k2 = S.kmax[1];
  for (int w = lane; w < nsite * 3; w += 32) {
    int st = w / 3, ax = w % 3;
    double f[3];
    frac_coords(S.cell, M.x[st], M.y[st], M.z[st], f);
    int off = st * stride + (ax == 0 ? 0 : (ax == 1 ? k1 + 1 : k1 + k2 + 2));
    axis_phases(f[ax], S.kmax[ax], reinterpret_cast<double2*>(tabv) + off);
  }
}

// Lane 0 of warp 0: the serial part of a move's set-up (gcmc.f:594-847): the move count and
// the 400-move checks, species and move choice, step-size adaptation, the counters, and every
// random number of the trial in the reference's order (utility_pack.f:2545-3000), which
// select_move leaves in M.r for the warp to build the trial sites from.
template <bool kProf>
__device__ __noinline__ void select_move(ChainDev& C, const SysConst& Y, MoveSmem& M) {
  if (kProf) C.prof[7] -= clock64();
  M.mj_action = 0;
  const bool second = M.mj_stage == 1;  // the second jump of a multi-jump: no count or selection
  if (!second) {
    M.mj_first = 0;  // a new move: no molecule to avoid
    C.gcmccount++;
    if (C.gcmccount % 400 == 0) check400(C, Y);
  }
  DuniLocal R(C.rng);  // written back before every return
  int g = M.g, mtype = kMultiJump;
  if (second) {
    M.mj_stage = 2;
  } else {
  const int ng = Y.nspecies;
  g = 0;
  if (ng > 1) g = (int)floor(R.next() * ng);
  double randmov = R.next();
  const double* c = C.mvcum[g];
  if (randmov < c[0]) mtype = kInsert;
  else if (randmov < c[1]) mtype = kDelete;
  else if (randmov < c[2]) mtype = kDisplace;
  else if (randmov < c[3]) mtype = kJump;
  else if (randmov < c[5]) mtype = kNoop;  // flex, swap (gcmc.f:1789-1795)
  else if (randmov < c[6]) mtype = kTranslate;
  else if (randmov < c[7]) mtype = kRotate;
  else if (randmov < c[8]) mtype = kMultiJump;
  else mtype = kDisplace;
  const int nmols = C.nmol[g];
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
  if (nmols == 0 || (nmols == 1 && mtype == kMultiJump)) mtype = kInsert;  // gcmc.f:837-847
  if (mtype == kMultiJump) {
    C.jump_count++;
    M.mj_stage = 1;
    M.mj_first = 0;
    M.mj_energy0 = C.energy[g];
  }
  }
  const SpeciesConst& P = Y.sp[g];
  const int ns = P.nsite, nmols = C.nmol[g];
  if (kProf) C.prof[7] += clock64();  // minus the stamp taken at entry: selection + adaptation
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
  M.rande_drawn = 0;
  double* r = M.r;
  if (mtype == kInsert) {
    C.ins_count++;
    if ((C.totatm - C.framatm) + ns >= C.maxguest || (nmols + 1) * ns > C.seg_cap[g]) {
      C.status = 75;
      R.store(C.rng);
      return;
    }
    for (int i = 0; i < 7; i++) r[i] = R.next();
    M.nnew = ns;
    for (int i = 0; i < ns; i++) C.numtyp[P.type[i]]++;
    M.need_lrc = 1;
  } else if (mtype == kDelete) {
    C.del_count++;
    int randchoice = (int)floor(R.next() * nmols) + 1;
    M.randchoice = randchoice;
    M.mol = randchoice - 1;
    M.ex_lo = C.seg_off[g] + M.mol * ns;
    M.ex_hi = M.ex_lo + ns;
    M.nold = ns;
    for (int i = 0; i < ns; i++) C.numtyp[P.type[i]]--;
    M.need_lrc = 1;
  } else if (mtype == kJump || mtype == kMultiJump) {
    // long jump (gcmc.f:1389-1547): the choice first, then the seven draws of random_jump; the
    // second jump of a multi-jump draws until it hits a molecule other than the first
    if (mtype == kJump) C.jump_count++;
    int randchoice;
    do {
      randchoice = (int)floor(R.next() * nmols) + 1;
    } while (randchoice == M.mj_first);
    if (mtype == kMultiJump && M.mj_stage == 1) M.mj_first = randchoice;
    M.randchoice = randchoice;
    M.mol = randchoice - 1;
    M.ex_lo = C.seg_off[g] + M.mol * ns;
    M.ex_hi = M.ex_lo + ns;
    for (int i = 0; i < 7; i++) r[i] = R.next();
    M.nold = ns;
    M.nnew = ns;
  } else if (mtype == kNoop) {
    // nothing moves; no sites, no draws beyond the move choice
  } else {
    if (mtype == kTranslate) {
      C.tran_count[g]++;
      r[0] = R.next();
      r[1] = R.next();
      r[2] = R.next();
      r[3] = r[4] = r[5] = r[6] = 0.0;
      M.dis_delr = C.tran_delr[g];
      M.dis_rot = 0.0;
    } else if (mtype == kRotate) {
      C.rota_count++;
      r[0] = r[1] = r[2] = 0.5;
      for (int i = 3; i < 7; i++) r[i] = R.next();
      M.dis_delr = 0.0;
      M.dis_rot = C.rota_rotangle;
    } else {
      C.disp_count[g]++;
      for (int i = 0; i < 7; i++) r[i] = R.next();
      M.dis_delr = C.delrdisp[g];
      M.dis_rot = C.rotangle;
    }
    int randchoice = (int)floor(R.next() * nmols) + 1;
    M.randchoice = randchoice;
    M.mol = randchoice - 1;
    M.ex_lo = C.seg_off[g] + M.mol * ns;
    M.ex_hi = M.ex_lo + ns;
    M.nold = ns;
    M.nnew = ns;
  }
  R.store(C.rng);
}

// ------------------------------------------------------------------ the trial sites, one lane each
// The trial generators of fmc_common.h restated for a warp: lane i holds site i, so the moved
// molecule's sites load at once and each site takes the same arithmetic as there; the mass centre
// sums run over the sites in order in every lane (gathered by shuffles), so every lane holds the
// same centre.
__device__ __forceinline__ void com_lanes(const double* mass, int n, double x, double y, double z, double* c) {
  double w = 0.0, sx = 0.0, sy = 0.0, sz = 0.0;
  for (int j = 0; j < n; j++) {
    const double xj = __shfl_sync(0xffffffffu, x, j), yj = __shfl_sync(0xffffffffu, y, j),
                 zj = __shfl_sync(0xffffffffu, z, j);
    w = w + mass[j];
    sx = sx + xj * mass[j];
    sy = sy + yj * mass[j];
    sz = sz + zj * mass[j];
  }
  c[0] = sx / w;
  c[1] = sy / w;
  c[2] = sz / w;
}

// One site rotated by quaternion q (rotate_sites' matrix).
__device__ __forceinline__ void rotate_site(const double q[4], double& x, double& y, double& z) {
  const double q1 = q[0], q2 = q[1], q3 = q[2], q4 = q[3];
  const double Q0 = 2.0 * q2 * q2 + 2.0 * q1 * q1 - 1.0, Q1 = 2.0 * q2 * q3 - 2.0 * q1 * q4;
  const double Q2 = 2.0 * q2 * q4 + 2.0 * q1 * q3, Q3 = 2.0 * q2 * q3 + 2.0 * q1 * q4;
  const double Q4 = 2.0 * q1 * q1 + 2.0 * q3 * q3 - 1.0, Q5 = 2.0 * q3 * q4 - 2.0 * q1 * q2;
  const double Q6 = 2.0 * q2 * q4 - 2.0 * q1 * q3, Q7 = 2.0 * q3 * q4 + 2.0 * q1 * q2;
  const double Q8 = 2.0 * q4 * q4 + 2.0 * q1 * q1 - 1.0;
  const double tx = Q0 * x + Q1 * y + Q2 * z;
  const double ty = Q3 * x + Q4 * y + Q5 * z;
  const double tz = Q6 * x + Q7 * y + Q8 * z;
  x = tx;
  y = ty;
  z = tz;
}

// Warp 0, after select_move: the trial sites (old sites read from the chain, new ones built by
// random_ins / random_disp + random_rot / random_jump), their charges and types, their voxel lists
// and the real-space work list, then their phase tables (ewald.f:95-137).
template <bool kProf>
__device__ __noinline__ void build_trial(ChainDev& C, const SysConst& Y, const DevSystem& S, MoveSmem& M, void* tab,
                                         int stride, int lane) {
  if (kProf && lane == 0) C.prof[8] -= clock64();
  const int mtype = M.mtype, ns = M.ns, nold = M.nold, nnew = M.nnew, nseg = Y.nspecies;
  const SpeciesConst& P = Y.sp[M.g];
  const bool mine = lane < ns;
  double ox = 0.0, oy = 0.0, oz = 0.0, nx = 0.0, ny = 0.0, nz = 0.0;
  int vb_old = 0, vl_old = 0;
  if (nold && mine) {
    const double4 a = C.gsite[M.ex_lo + lane];
    ox = a.x;
    oy = a.y;
    oz = a.z;
    // the old site's voxel list, looked up while the trial geometry is computed
    const int v = voxel_of(S, ox, oy, oz);
    vb_old = S.vox_off[v];
    vl_old = S.vox_off[v + 1] - vb_old;
  }
  const double* r = M.r;
  const double* h = S.cell.h;
  if (mtype == kInsert) {
    // random_ins (utility_pack.f:2545-2650): template rotated, centred at fractional (r0, r1, r2)
    const double xc = r[0] * h[0] + r[1] * h[3] + r[2] * h[6];
    const double yc = r[0] * h[1] + r[1] * h[4] + r[2] * h[7];
    const double zc = r[0] * h[2] + r[1] * h[5] + r[2] * h[8];
    double q[4];
    axis_angle_quat(r[3] * 2.0 * kPi, r[4], r[5], r[6], q);
    if (mine) {
      nx = P.tx[lane];
      ny = P.ty[lane];
      nz = P.tz[lane];
      rotate_site(q, nx, ny, nz);
      nx = nx + xc;
      ny = ny + yc;
      nz = nz + zc;
    }
  } else if (mtype == kJump || mtype == kMultiJump) {
    // random_jump: the mass centre moved to fractional (r0, r1, r2), a new orientation about it
    double xd = r[0] * h[0] + r[1] * h[3] + r[2] * h[6];
    double yd = r[0] * h[1] + r[1] * h[4] + r[2] * h[7];
    double zd = r[0] * h[2] + r[1] * h[5] + r[2] * h[8];
    double cm[3];
    com_lanes(P.mass, ns, ox, oy, oz, cm);
    xd = xd - cm[0];
    yd = yd - cm[1];
    zd = zd - cm[2];
    nx = xd + ox;
    ny = yd + oy;
    nz = zd + oz;
    com_lanes(P.mass, ns, nx, ny, nz, cm);
    nx = nx - cm[0];
    ny = ny - cm[1];
    nz = nz - cm[2];
    double q[4];
    axis_angle_quat(r[3] * (8.0 * atan(1.0)), r[4], r[5], r[6], q);
    rotate_site(q, nx, ny, nz);
    nx = nx + cm[0];
    ny = ny + cm[1];
    nz = nz + cm[2];
  } else if (mtype == kDisplace || mtype == kTranslate || mtype == kRotate) {
    // random_disp + random_rot (utility_pack.f:2679-2763, 2929-3000)
    const double half = M.dis_delr * 0.5;
    const double dx = (2.0 * r[0] - 1.0) * half, dy = (2.0 * r[1] - 1.0) * half, dz = (2.0 * r[2] - 1.0) * half;
    nx = dx + ox;
    ny = dy + oy;
    nz = dz + oz;
    double cm[3];
    com_lanes(P.mass, ns, nx, ny, nz, cm);
    const double* rh = S.cell.rh;
    double fx = rh[0] * cm[0] + rh[3] * cm[1] + rh[6] * cm[2];
    double fy = rh[1] * cm[0] + rh[4] * cm[1] + rh[7] * cm[2];
    double fz = rh[2] * cm[0] + rh[5] * cm[1] + rh[8] * cm[2];
    fx = fx - floor(fx);
    fy = fy - floor(fy);
    fz = fz - floor(fz);
    const double wx = h[0] * fx + h[3] * fy + h[6] * fz;
    const double wy = h[1] * fx + h[4] * fy + h[7] * fz;
    const double wz = h[2] * fx + h[5] * fy + h[8] * fz;
    const double shx = wx - cm[0], shy = wy - cm[1], shz = wz - cm[2];
    nx = nx + shx - wx;
    ny = ny + shy - wy;
    nz = nz + shz - wz;
    double q[4];
    axis_angle_quat(r[3] * M.dis_rot, r[4], r[5], r[6], q);
    rotate_site(q, nx, ny, nz);
    nx = nx + wx;
    ny = ny + wy;
    nz = nz + wz;
  }
  // the work list: each trial site's voxel list, then every guest site
  if (mine && nold) {
    M.x[lane] = ox;
    M.y[lane] = oy;
    M.z[lane] = oz;
    M.q[lane] = P.q[lane];
    M.type[lane] = P.type[lane];
    M.vb[lane] = vb_old;
    M.vl[lane] = vl_old;
  }
  if (mine && nnew) {
    const int st = nold + lane;
    M.x[st] = nx;
    M.y[st] = ny;
    M.z[st] = nz;
    M.q[st] = P.q[lane];
    M.type[st] = P.type[lane];
    const int v = voxel_of(S, nx, ny, nz);
    M.vb[st] = S.vox_off[v];
    M.vl[st] = S.vox_off[v + 1] - S.vox_off[v];
  }
  __syncwarp();
  build_phases(S, M, tab, stride, lane);
  // work-list prefix over the sites: each site's voxel list plus every guest site (warp scan)
  int gt = 0;
  for (int g = 0; g < nseg; g++) gt += C.nmol[g] * Y.sp[g].nsite;
  int w = lane < nold + nnew ? M.vl[lane] + gt : 0;
  for (int o = 1; o < 32; o <<= 1) {
    const int u = __shfl_up_sync(0xffffffffu, w, o);
    if (lane >= o) w += u;
  }
  if (lane < nold + nnew) M.pre[lane + 1] = w;
  if (lane == 0) {
    M.pre[0] = 0;
    int acc = 0;
    M.gpre[0] = 0;
    for (int g = 0; g < nseg; g++) {
      acc += C.nmol[g] * Y.sp[g].nsite;
      M.gpre[g + 1] = acc;
    }
    if (kProf) C.prof[8] += clock64();
  }
}

// Real-space sums of one pass: every (site, candidate) pair, compiled per boundary condition so
// the hot loop holds one minimum-image form.  Deeper unrolling (2-8 candidates per trip) was
// measured slower: the larger loop costs more in instruction fetch than it hides in latency.
template <int kImcon, int NT, int CPT>
__device__ __noinline__ void real_space(const DevSystem& S, const ChainDev& C, const MoveSmem& M, int nseg,
                                        const int* prow_s, int nt1, double* vout) {
  const int tid = threadIdx.x, nsite = M.nold + M.nnew, nold = M.nold, mtype = M.mtype;
  double v1 = vout[1], v2 = vout[2];
  const bool sub_old = (mtype != kInsert && mtype != kDelete);
  const int T = M.pre[nsite];
  // a thread takes candidates tid, tid + NT, tid + 2 NT, ... and adds them in that order;
  // CPT candidates per loop trip, the next trip's loads issued before this one is evaluated
  // (the pair's accumulation is written out in each loop: passing the candidate to a helper
  // made ptxas spill in this loop)
  if (CPT == 1) {
    int s_next = 0;
    Cand pre = fetch_candidate(S, C, M, nseg, tid, s_next);
    for (int base = tid; base < T; base += NT) {
      const Cand c = pre;
      pre = fetch_candidate(S, C, M, nseg, base + NT, s_next);
      if (!c.live) continue;
      const int st = c.site;
      const int row = prow_s[M.type[st] * nt1 + c.type];
      double ec = 0.0, ev = 0.0;
      pair_energy<kImcon>(S, M.x[st] - c.a.x, M.y[st] - c.a.y, M.z[st] - c.a.z, M.q[st] * kR4pie0, c.a.w, row, ec,
                          ev);
      if (sub_old && st < nold) {
        v1 -= ec;
        v2 -= ev;
      } else {
        v1 += ec;
        v2 += ev;
      }
    }
  } else {
    int s0 = 0, s1 = 0;
    Cand p0 = fetch_candidate(S, C, M, nseg, tid, s0);
    Cand p1 = fetch_candidate(S, C, M, nseg, tid + NT, s1);
    for (int base = tid; base < T; base += 2 * NT) {
      const Cand c0 = p0, c1 = p1;
      p0 = fetch_candidate(S, C, M, nseg, base + 2 * NT, s0);
      p1 = fetch_candidate(S, C, M, nseg, base + 3 * NT, s1);
      if (c0.live) {
        const int st = c0.site;
        const int row = prow_s[M.type[st] * nt1 + c0.type];
        double ec = 0.0, ev = 0.0;
        pair_energy<kImcon>(S, M.x[st] - c0.a.x, M.y[st] - c0.a.y, M.z[st] - c0.a.z, M.q[st] * kR4pie0, c0.a.w, row,
                            ec, ev);
        if (sub_old && st < nold) {
          v1 -= ec;
          v2 -= ev;
        } else {
          v1 += ec;
          v2 += ev;
        }
      }
      if (c1.live) {
        const int st = c1.site;
        const int row = prow_s[M.type[st] * nt1 + c1.type];
        double ec = 0.0, ev = 0.0;
        pair_energy<kImcon>(S, M.x[st] - c1.a.x, M.y[st] - c1.a.y, M.z[st] - c1.a.z, M.q[st] * kR4pie0, c1.a.w, row,
                            ec, ev);
        if (sub_old && st < nold) {
          v1 -= ec;
          v2 -= ev;
        } else {
          v1 += ec;
          v2 += ev;
        }
      }
    }
  }
  vout[1] = v1;
  vout[2] = v2;
}

// All threads: this thread's share of the reciprocal sum (v[0] = sum akk*d|S|^2) and of the
// real-space pairs (v[1] ewld2, v[2] vdw); S_new goes to Sn.
// One k-vector's change: S_new(k) from S(k) and the trial sites' phases; returns
// akk (|S_new|^2 - |S_old|^2).
__device__ __forceinline__ double recip_term(int k, const MoveSmem& M, const int* kp, const double* ak,
                                             const double2* Sk, double2* Sn, const double2* tb, int stride, int k1,
                                             int k2) {
  const int nsite = M.nold + M.nnew, nold = M.nold, mtype = M.mtype;
  int l, m, n;
  kunpack(kp[k], l, m, n);
  int am = m < 0 ? -m : m, an = n < 0 ? -n : n;
  double2 so = Sk[k], sn;
  double2 aold = make_double2(0.0, 0.0), anew = make_double2(0.0, 0.0);
  for (int st = 0; st < nsite; st++) {
    const double2* t = tb + st * stride;
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
  if (mtype == kInsert)
    sn = make_double2(anew.x + so.x, anew.y + so.y);
  else if (mtype == kDelete)
    sn = make_double2(so.x - aold.x, so.y - aold.y);
  else
    sn = make_double2((so.x - aold.x) + anew.x, (so.y - aold.y) + anew.y);
  Sn[k] = sn;
  return ak[k] * (sn.x * sn.x + sn.y * sn.y - so.x * so.x - so.y * so.y);
}

// All threads: this thread's share of the reciprocal sum (v[0] = sum akk*d|S|^2) and of the
// real-space pairs (v[1] ewld2, v[2] vdw); S_new goes to Sn.  A thread takes k-vectors tid,
// tid + NT, ... and adds their terms in that order, KPT of them per trip.
template <int NT, int KPT, int CPT>
__device__ __noinline__ void sums(const DevSystem& S, const ChainDev& C, const MoveSmem& M, int nseg, const int* prow_s,
                                  int nt1, const int* kp, const double* ak, const double2* Sk, double2* Sn,
                                  const void* tabv, int stride, double* v) {
  const int tid = threadIdx.x, K = S.K, k1 = S.kmax[0], k2 = S.kmax[1];
  const double2* tb = reinterpret_cast<const double2*>(tabv);
  if (KPT == 1) {
    for (int k = tid; k < K; k += NT) v[0] += recip_term(k, M, kp, ak, Sk, Sn, tb, stride, k1, k2);
  } else {
    int k = tid;
    for (; k + NT < K; k += 2 * NT) {  // two independent k-vectors in flight, added in order
      v[0] += recip_term(k, M, kp, ak, Sk, Sn, tb, stride, k1, k2);
      v[0] += recip_term(k + NT, M, kp, ak, Sk, Sn, tb, stride, k1, k2);
    }
    if (k < K) v[0] += recip_term(k, M, kp, ak, Sk, Sn, tb, stride, k1, k2);
  }
  // real space, per boundary condition
  if (S.cell.imcon == 1) real_space<1, NT, CPT>(S, C, M, nseg, prow_s, nt1, v);
  else if (S.cell.imcon == 2) real_space<2, NT, CPT>(S, C, M, nseg, prow_s, nt1, v);
  else if (S.cell.imcon == 3) real_space<3, NT, CPT>(S, C, M, nseg, prow_s, nt1, v);
  // the half-shift cells and the slab share one instantiation that reads the boundary condition
  // from the cell: each compiled copy of this loop costs instruction cache (one per cell kind
  // cost 8%)
  else real_space<-1, NT, CPT>(S, C, M, nseg, prow_s, nt1, v);
}

// All threads, in production: storeprob (utility_pack.f:496-561) for the chain's state after the
// move, one guest molecule per thread, weights added to the plots' fixed-point grids.
__device__ __noinline__ void prob_store(const SysConst& Y, const ChainDev& C) {
  const int na = Y.ngrid[0], nb = Y.ngrid[1], nc = Y.ngrid[2];
  const long long cells = (long long)na * nb * nc;
  for (int g = 0; g < Y.nspecies; g++) {
    const SpeciesConst& P = Y.sp[g];
    const int ns = P.nsite, nmol = C.nmol[g];
    for (int m = threadIdx.x; m < nmol; m += blockDim.x) {
      double x[kBatchMaxSites], y[kBatchMaxSites], z[kBatchMaxSites];
      const double4* site = C.gsite + C.seg_off[g] + m * ns;
      for (int i = 0; i < ns; i++) {
        double4 a = site[i];
        x[i] = a.x;
        y[i] = a.y;
        z[i] = a.z;
      }
      double c[3], fc[3];
      centre_of_mass(P.mass, ns, x, y, z, 1, c);
      frac_wrap(Y.S.cell.rh, c[0], c[1], c[2], fc);
      for (int ip = 0; ip < Y.nplots; ip++) {
        if (Y.plot_guest[ip] != g) continue;
        unsigned long long* grid = C.prob + ip * cells;
        auto add = [grid](long long i, double w) {
          atomicAdd(grid + i, (unsigned long long)llrint(w * 4294967296.0));
        };
        for (int j = 0; j < Y.plot_nsite[ip]; j++) {
          const int s = Y.plot_site[ip][j];
          if (s == 0) {
            equitable_bin(na, nb, nc, fc[0], fc[1], fc[2], add);
          } else {
            double f[3];
            frac_wrap(Y.S.cell.rh, x[s - 1], y[s - 1], z[s - 1], f);
            equitable_bin(na, nb, nc, f[0], f[1], f[2], add);
          }
        }
      }
    }
  }
}

template <bool kProf, int NT, int KPT, int CPT>
__global__ void __launch_bounds__(NT, NT <= 128 ? 4 : (NT <= 256 ? 2 : 1)) fmc_batch_kernel(BatchLaunch L,
                                                                                           int tab_stride) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ ChainDev C;
  __shared__ MoveSmem M;
  __shared__ SysConst Ysm;
  __shared__ double red[32 * 3];
  __shared__ int prow_s[(kBatchMaxTypes + 1) * (kBatchMaxTypes + 1)];
  DevSystem& S = Ysm.S;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if ((int)blockIdx.x >= L.nchains) return;
  const int cidx = L.order ? L.order[blockIdx.x] : (int)blockIdx.x;  // the chain this CTA runs
  if (!L.chains[cidx].active) return;
  const long long t_start = L.timing && tid == 0 ? global_ns() : 0;
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
  void* tab = reinterpret_cast<void*>(kp + ((Kmax + 3) & ~3));
  for (int k = tid; k < K; k += blockDim.x) {
    Sk[k] = C.sk[k];
    ak[k] = S.akk[k];
    kp[k] = S.kpack[k];
  }
  const int stride = S.kmax[0] + S.kmax[1] + S.kmax[2] + 3;
  (void)tab_stride;
  __syncthreads();
  long long t0 = 0, t1 = 0;
  constexpr bool prof = kProf;
  // a chain ends after the move on which its deck's equilibration + production budget ran
  // out (the reference's do-while(lgchk) loop, gcmc.f:589-736), or at its move budget
  long long nmoves = C.lgchk ? L.moves : 0;
  if (C.budget > 0) nmoves = min(nmoves, C.budget - C.moves_done);
  if (tid == 0) M.mj_stage = 0;
  bool pending = false;  // the first half of a multi-jump ended the last trip; the move goes on
  for (int mv = 0; mv < nmoves;) {
    if (prof && tid == 0) t0 = clock64();
    if (warp == 0) {
      if (lane == 0) select_move<kProf>(C, Y, M);
      __syncwarp();
      // warp 1 may read select_move's results now (named barrier 1: warps 0 and 1)
      asm volatile("bar.arrive 1, 64;" ::: "memory");
      if (!C.status) build_trial<kProf>(C, Y, S, M, tab, stride, lane);
    } else if (warp == 1) {
      asm volatile("bar.sync 1, 64;" ::: "memory");
      if (M.need_lrc && !C.status) lrc_warp(C, Y, M, lane);
    }
    __syncthreads();
    if (prof && tid == 0) {
      t1 = clock64();
      C.prof[0] += t1 - t0;
      t0 = t1;
    }
    if (C.status) break;
    const bool last = !C.lgchk;  // lane 0 of warp 0 writes lgchk only in select_move
    double v[3] = {0.0, 0.0, 0.0};
    sums<NT, KPT, CPT>(S, C, M, nseg, prow_s, nt1, kp, ak, Sk, Sn, tab, stride, v);
    if (prof && tid == 0) C.prof[6] += clock64() - t0;
    block_sum<3>(v, red);
    if (prof && tid == 0) {
      t1 = clock64();
      C.prof[2] += t1 - t0;
      t0 = t1;
    }
    if (tid == 0) {
      assemble(Y, M, v);
      decide(C, Y, M);
    }
    __syncthreads();
    if (tid == 0) bookkeep(C, Y, M, L.trace ? L.trace + (size_t)cidx * L.moves + mv : nullptr);
    __syncthreads();
    if (prof && tid == 0) {
      t1 = clock64();
      C.prof[3] += t1 - t0;
      t0 = t1;
    }
    if (M.mj_action == 1)  // park S(k) before the first jump of a multi-jump is committed
      for (int k = tid; k < K; k += blockDim.x) C.sk[k] = Sk[k];
    if (M.mj_action == 2) {  // rejected multi-jump: S(k) and the first molecule as they were
      for (int k = tid; k < K; k += blockDim.x) Sk[k] = C.sk[k];
      if (tid < M.ns)
        C.gsite[M.mj_lo + tid] =
            make_double4(M.mj_old[3 * tid], M.mj_old[3 * tid + 1], M.mj_old[3 * tid + 2], Y.sp[M.g].q[tid]);
    }
    if (M.accepted) {
      for (int k = tid; k < K; k += blockDim.x) Sk[k] = Sn[k];
      const int ns = M.ns, mtype = M.mtype;
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
    // read before the barrier: thread 0 may change these in the next select_move
    pending = M.mj_stage == 1;
    const bool store = Y.nplots && C.production && !pending;
    __syncthreads();
    if (prof && tid == 0) C.prof[4] += clock64() - t0;
    if (store) prob_store(Y, C);  // every production move (gcmc.f:1929-1931)
    if (pending) continue;
    if (last) break;
    mv++;
  }
  for (int k = tid; k < K; k += blockDim.x) C.sk[k] = Sk[k];
  if (tid == 0 && L.retire_finished && ((C.budget > 0 && C.moves_done >= C.budget) || !C.lgchk || C.status))
    C.active = 0;
  __syncthreads();
  {
    const int* src = reinterpret_cast<const int*>(&C);
    int* dst = reinterpret_cast<int*>(&L.chains[cidx]);
    for (int i = tid; i < (int)(sizeof(ChainDev) / sizeof(int)); i += blockDim.x) dst[i] = src[i];
  }
  if (L.timing && tid == 0) {
    unsigned sm;
    asm volatile("mov.u32 %0, %%smid;" : "=r"(sm));
    L.timing[3 * cidx] = t_start;
    L.timing[3 * cidx + 1] = global_ns();
    L.timing[3 * cidx + 2] = sm;
  }
}

}  // namespace

int batch_smem_bytes(int kmax_K, int tab_sites, int tab_stride) {
  return kmax_K * (int)(2 * sizeof(double2) + sizeof(double)) + ((kmax_K + 3) & ~3) * (int)sizeof(int) +
         tab_sites * tab_stride * (int)sizeof(double2);
}

namespace {
using BatchKernel = void (*)(BatchLaunch, int);
// the kernel of each tile of kBatchTiles, in the same order
constexpr BatchKernel kTileKernels[kNumBatchTiles] = {
    fmc_batch_kernel<false, 256, 1, 1>, fmc_batch_kernel<false, 256, 2, 1>, fmc_batch_kernel<false, 256, 1, 2>,
    fmc_batch_kernel<false, 256, 2, 2>, fmc_batch_kernel<false, 128, 1, 1>, fmc_batch_kernel<false, 128, 2, 1>,
    fmc_batch_kernel<false, 128, 1, 2>, fmc_batch_kernel<false, 128, 2, 2>, fmc_batch_kernel<false, 384, 1, 1>,
    fmc_batch_kernel<false, 384, 2, 1>, fmc_batch_kernel<false, 384, 1, 2>, fmc_batch_kernel<false, 384, 2, 2>};
constexpr BatchKernel kProfKernel = fmc_batch_kernel<true, 256, 1, 1>;
}  // namespace

// The dynamic shared-memory limit belongs to the kernel, shared by every batch and server of the
// process on the current device: it only ever rises, so that opening a batch with smaller tables
// cannot make the launches of one opened before it (with larger tables) exceed the limit.
cudaError_t configure_batch_kernel(int smem_bytes) {
  static std::mutex mu;
  static std::map<int, int> limit;  // device -> the limit set on it
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lk(mu);
  int& have = limit[dev];
  if (smem_bytes <= have) return cudaSuccess;
  e = cudaFuncSetAttribute(kProfKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_bytes);
  for (int t = 0; t < kNumBatchTiles && e == cudaSuccess; t++)
    e = cudaFuncSetAttribute(kTileKernels[t], cudaFuncAttributeMaxDynamicSharedMemorySize, smem_bytes);
  if (e == cudaSuccess) have = smem_bytes;
  return e;
}

cudaError_t launch_batch(const BatchLaunch& L, int smem_bytes, int tab_stride, cudaStream_t st) {
  if (L.tile < 0 || L.tile >= kNumBatchTiles || (L.profile && L.tile != 0)) return cudaErrorInvalidValue;
  const BatchKernel k = L.profile ? kProfKernel : kTileKernels[L.tile];
  k<<<L.nchains, kBatchTiles[L.tile].threads, smem_bytes, st>>>(L, tab_stride);
  return cudaGetLastError();
}

}  // namespace fmc
