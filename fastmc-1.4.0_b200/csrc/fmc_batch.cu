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
  int commit_lo, seg_end, ns, randchoice;
  double delrc, rande;
  double x[2 * kBatchMaxSites], y[2 * kBatchMaxSites], z[2 * kBatchMaxSites], q[2 * kBatchMaxSites];
  int type[2 * kBatchMaxSites];
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
__device__ __noinline__ void move_begin(ChainDev& C, const SysConst& Y, MoveSmem& M) {
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
  M.mtype = mtype;
  M.g = g;
  M.ns = ns;
  M.mol = -1;
  M.randchoice = 0;
  M.ex_lo = M.ex_hi = -1;
  M.nold = M.nnew = 0;
  M.delrc = 0.0;
  M.rande = -1.0;
  if (mtype < 0) {
    C.status = 3;
    return;
  }
  double* x = M.x;
  double* y = M.y;
  double* z = M.z;
  if (mtype == kInsert) {
    C.ins_count++;
    if ((C.totatm - C.framatm) + ns >= C.maxguest || (nmols + 1) * ns > C.seg_cap[g]) {
      C.status = 75;
      return;
    }
    double r[7];
    for (int i = 0; i < 7; i++) r[i] = duni_next(C.rng);
    trial_insert(Y.S.cell, P.tx, P.ty, P.tz, ns, r, x, y, z);
    M.nnew = ns;
    for (int i = 0; i < ns; i++) C.numtyp[P.type[i]]++;
    M.delrc = lrc_device(Y, C.numtyp) - C.elrc;
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
    M.delrc = lrc_device(Y, C.numtyp) - C.elrc;
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
    trial_displace(Y.S.cell, P.mass, ns, dis_delr, dis_rot, r, x + ns, y + ns, z + ns);
    M.nold = ns;
    M.nnew = ns;
  }
  for (int i = 0; i < M.nold + M.nnew; i++) {
    int s = i < M.nold ? i : i - M.nold;
    M.q[i] = P.q[s];
    M.type[i] = P.type[s];
  }
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

__global__ void __launch_bounds__(kBatchThreads, 2) fmc_batch_kernel(BatchLaunch L, int tab_stride) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ ChainDev C;
  __shared__ MoveSmem M;
  __shared__ DevSystem S;
  __shared__ double red[32 * 3];
  const int tid = threadIdx.x, cidx = blockIdx.x;
  if (cidx >= L.nchains) return;
  {
    const int* src = reinterpret_cast<const int*>(&L.chains[cidx]);
    int* dst = reinterpret_cast<int*>(&C);
    for (int i = tid; i < (int)(sizeof(ChainDev) / sizeof(int)); i += blockDim.x) dst[i] = src[i];
  }
  __syncthreads();
  const SysConst& Y = L.systems[C.sys];
  if (tid == 0) S = Y.S;
  __syncthreads();
  const int K = S.K, Kmax = L.kmax_smem;
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
  for (int mv = 0; mv < L.moves; mv++) {
    if (tid == 0) move_begin(C, Y, M);
    __syncthreads();
    if (C.status) break;
    const int nsite = M.nold + M.nnew;
    for (int w = tid; w < nsite * 3; w += blockDim.x) {
      int s = w / 3, ax = w % 3;
      double f[3];
      frac_coords(S.cell, M.x[s], M.y[s], M.z[s], f);
      axis_phases(f[ax], S.kmax[ax], tab + s * stride + (ax == 0 ? 0 : (ax == 1 ? k1 + 1 : k1 + k2 + 2)));
    }
    __syncthreads();
    double v[3] = {0.0, 0.0, 0.0};
    const int mtype = M.mtype, nold = M.nold;
    for (int k = tid; k < K; k += blockDim.x) {
      int l, m, n;
      kunpack(kp[k], l, m, n);
      int am = m < 0 ? -m : m, an = n < 0 ? -n : n;
      double2 aold = make_double2(0.0, 0.0), anew = make_double2(0.0, 0.0);
      for (int s = 0; s < nsite; s++) {
        const double2* t = tab + s * stride;
        double2 c = m >= 0 ? cmul(t[l], t[k1 + 1 + am]) : cmulc(t[l], t[k1 + 1 + am]);
        c = n >= 0 ? cmul(c, t[k1 + k2 + 2 + an]) : cmulc(c, t[k1 + k2 + 2 + an]);
        double q = M.q[s];
        if (s < nold) {
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
    GuestView G;
    G.site = C.gsite;
    G.type = C.gtype;
    G.nseg = Y.nspecies;
    for (int g = 0; g < kMaxGuestTypes; g++) {
      G.seg_off[g] = C.seg_off[g];
      G.seg_len[g] = g < Y.nspecies ? C.nmol[g] * Y.sp[g].nsite : 0;
    }
    const bool sub_old = (mtype != kInsert && mtype != kDelete);
    for (int s = 0; s < nsite; s++) {
      double ecf = 0.0, evf = 0.0, ecg = 0.0, evg = 0.0;
      site_partial(S, G, M.x[s], M.y[s], M.z[s], M.q[s], M.type[s], M.ex_lo, M.ex_hi, tid, blockDim.x, ecf, evf,
                   ecg, evg);
      if (sub_old && s < nold) {
        v[1] -= ecf + ecg;
        v[2] -= evf + evg;
      } else {
        v[1] += ecf + ecg;
        v[2] += evf + evg;
      }
    }
    block_sum<3>(v, red);
    if (tid == 0) move_end(C, Y, M, v, L.trace ? L.trace + (size_t)cidx * L.moves + mv : nullptr);
    __syncthreads();
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
        int s = (mtype == kInsert) ? tid : ns + tid;
        C.gsite[M.commit_lo + tid] = make_double4(M.x[s], M.y[s], M.z[s], M.q[s]);
        C.gtype[M.commit_lo + tid] = M.type[s];
      }
    }
    __syncthreads();
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
