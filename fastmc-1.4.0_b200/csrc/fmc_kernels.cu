// FP64 kernels of the plain (one trial per launch) GPU path.
//
// fmc_pass_kernel   : one launch per trial move.  Blocks [0, nbk) compute the reciprocal
//                     change over all K k-vectors (ewald1_guest, ewald.f:32-365): per-site
//                     axis phase tables in shared memory, one k-vector per thread, S_new to
//                     scratch, akk*(|S_new|^2-|S_old|^2) reduced per block.  Blocks [nbk, ...)
//                     compute the real-space erfc Coulomb + tabulated vdW energy of one
//                     trial site each (ewald2 + srfrce over the neighbour set that
//                     guestlistgen would build).  The last block to finish combines the
//                     block partials in a fixed order (deterministic) into {ewld1, ewld2, vdw}.
// fmc_commit_kernel : S(k) <- S_new and the guest-site array update of an accepted move.
// fmc_recip_*       : full S(k) of a set of atoms (ewald1, ewald.f:368-630).
// fmc_sp_kernel     : per-guest-site real-space energies for the single-point energy.
#include <cmath>
#include <cstddef>
#include <cstring>

#include "fmc_device.cuh"
#include "fmc_kernels.h"

namespace fmc {

constexpr int kPassThreads = 256;
static_assert(2 * kMaxPassSites <= kPassThreads, "the combine stages every site energy in one pass");

// A guest-site update by one block (all its threads): a delete removes [lo, lo+ns) and shifts
// the rest of the segment down in order; an insert writes at the segment end, a displacement
// over the molecule.
__device__ __forceinline__ void apply_commit(const PendingCommit& P, double4* site, int* type) {
  const int tid = threadIdx.x;
  if (P.op == kDelete) {
    const int ns = P.ns;
    for (int base = P.lo; base < P.seg_end - ns; base += blockDim.x) {
      const int i = base + tid;
      const bool act = i < P.seg_end - ns;
      double4 a = make_double4(0.0, 0.0, 0.0, 0.0);
      int t = 0;
      if (act) {
        a = site[i + ns];
        t = type[i + ns];
      }
      __syncthreads();
      if (act) {
        site[i] = a;
        type[i] = t;
      }
      __syncthreads();
    }
  } else if (tid < P.ns) {
    site[P.lo + tid] = P.site[tid];
    type[P.lo + tid] = P.type[tid];
  }
}

// ------------------------------------------------------------------------------ pass
// One block's share of a trial pass (block `blk` of `nblocks`): blocks [0, nbk) the reciprocal
// change of 256 k-vectors each, the next nsite blocks the real-space energy of one trial site
// each (further blocks idle), then the last block to finish combines the partials in a fixed
// order into {ewld1, ewld2, vdw}, publishes them with the sequence number and writes the pending
// guest-site update.  Returns (to every thread) whether this block was the last.
template <class Args>
__device__ __forceinline__ bool pass_block(const DevSystem& S, const GuestView& G, const Args& A, const double2* sk,
                                           double2* sk_new, const PassScratch& W, int blk, int nblocks,
                                           double2* sm_tab, double* red, double* comb, bool& am_last) {
  const int nsite = A.nold + A.nnew;
  const int nbk = A.nbk;
  const int tid = threadIdx.x;
  if (blk < nbk) {
    // ---- reciprocal space
    const int k1 = S.kmax[0], k2 = S.kmax[1], k3 = S.kmax[2];
    const int stride = (k1 + 1) + (k2 + 1) + (k3 + 1);
    for (int w = tid; w < nsite * 3; w += blockDim.x) {
      int s = w / 3, ax = w % 3;
      double f[3];
      frac_coords(S.cell, A.x[s], A.y[s], A.z[s], f);
      double2* t = sm_tab + s * stride + (ax == 0 ? 0 : (ax == 1 ? k1 + 1 : k1 + k2 + 2));
      axis_phases(f[ax], S.kmax[ax], t);
    }
    __syncthreads();
    double v[1] = {0.0};
    int k = blk * blockDim.x + tid;
    if (k < S.K) {
      int l, m, n;
      kunpack(S.kpack[k], l, m, n);
      int am = m < 0 ? -m : m, an = n < 0 ? -n : n;
      double2 aold = make_double2(0.0, 0.0), anew = make_double2(0.0, 0.0);
      for (int s = 0; s < nsite; s++) {
        const double2* t = sm_tab + s * stride;
        double2 e1 = t[l], e2 = t[k1 + 1 + am], e3 = t[k1 + k2 + 2 + an];
        double2 c = m >= 0 ? cmul(e1, e2) : cmulc(e1, e2);
        c = n >= 0 ? cmul(c, e3) : cmulc(c, e3);
        double q = A.q[s];
        if (s < A.nold) {
          aold.x += q * c.x;
          aold.y += q * c.y;
        } else {
          anew.x += q * c.x;
          anew.y += q * c.y;
        }
      }
      double2 so = sk[k], sn;
      if (A.move == kInsert)
        sn = make_double2(anew.x + so.x, anew.y + so.y);
      else if (A.move == kDelete)
        sn = make_double2(so.x - aold.x, so.y - aold.y);
      else
        sn = make_double2((so.x - aold.x) + anew.x, (so.y - aold.y) + anew.y);
      sk_new[k] = sn;
      v[0] = S.akk[k] * (sn.x * sn.x + sn.y * sn.y - so.x * so.x - so.y * so.y);
    }
    block_sum<1>(v, red);
    if (tid == 0) W.recip_part[blk] = v[0];
  } else if (A.do_real && blk - nbk < nsite) {
    // ---- real space of one trial site
    const int s = blk - nbk;
    double v[2] = {0.0, 0.0};
    double ec_fw = 0.0, ev_fw = 0.0, ec_g = 0.0, ev_g = 0.0;
    site_partial(S, G, A.pc, A.x[s], A.y[s], A.z[s], A.q[s], A.type[s], A.ex_lo, A.ex_hi, tid, blockDim.x, ec_fw,
                 ev_fw, ec_g, ev_g);
    v[0] = ec_g + ec_fw;
    v[1] = ev_g + ev_fw;
    block_sum<2>(v, red);
    if (tid == 0) {
      W.site_e[2 * s] = v[0];
      W.site_e[2 * s + 1] = v[1];
    }
  }
  // ---- last block combines in a fixed order: the partials are loaded by all its threads at
  // once and summed by thread 0 in block / site order
  if (tid == 0) {
    __threadfence();
    unsigned done = atomicAdd(W.counter, 1u);
    am_last = (done == (unsigned)nblocks - 1);
  }
  __syncthreads();
  if (!am_last) return false;
  __threadfence();
  double r = 0.0;
  for (int base = 0; base < nbk; base += kPassThreads) {
    if (base + tid < nbk) comb[tid] = ((volatile double*)W.recip_part)[base + tid];
    __syncthreads();
    if (tid == 0)
      for (int i = 0; i < kPassThreads && base + i < nbk; i++) r += comb[i];
    __syncthreads();
  }
  const int nse = A.do_real ? 2 * nsite : 0;  // <= 2 * kMaxPassSites <= kPassThreads
  if (tid < nse) comb[tid] = ((volatile double*)W.site_e)[tid];
  __syncthreads();
  if (tid == 0) {
    double ewld1 = S.recip_pref * r;
    if (A.move == kInsert) ewld1 = ewld1 + A.engsic;
    if (A.move == kDelete) ewld1 = ewld1 - A.engsic;
    double e2 = 0.0, ev = 0.0;
    const double* se = comb;
    for (int s = 0; s < (A.do_real ? nsite : 0); s++) {
      if (s < A.nold && A.move == kDisplace) {
        e2 = e2 - se[2 * s];
        ev = ev - se[2 * s + 1];
      } else {
        e2 = e2 + se[2 * s];
        ev = ev + se[2 * s + 1];
      }
    }
    W.result[0] = ewld1;
    W.result[1] = e2;
    W.result[2] = ev;
    __threadfence_system();  // the energies reach the host before the sequence number does
    ((volatile double*)W.result)[3] = A.seq;
    *W.counter = 0u;
  }
  // every block has read the guest sites: the last one writes the pending update
  if (A.pc.op) apply_commit(A.pc, W.gsite, W.gtype);
  return true;
}

template <int N>
__global__ void __launch_bounds__(kPassThreads) fmc_pass_kernel(DevSystem S, GuestView G, PassArgsT<N> A,
                                                                const double2* __restrict__ sk, double2* sk_new,
                                                                PassScratch W) {
  extern __shared__ double2 sm_tab[];
  __shared__ double red[32 * 2];
  __shared__ double comb[kPassThreads];
  __shared__ bool am_last;
  pass_block(S, G, A, sk, sk_new, W, (int)blockIdx.x, (int)gridDim.x, sm_tab, red, comb, am_last);
}

// ------------------------------------------------------------------------------ resident pass
// Every wait of the resident kernel is bounded on the device clock (%globaltimer, ns): block 0
// ends the kernel after `idle_ns` without a pass (the host passes the limit); the other blocks
// wait for block 0 up to 64 times as long, and for the previous pass's update up to kDoneNs:
// past either limit a block records why in host_words[1] and ends.
constexpr unsigned long long kDoneNs = 1000000000ULL;

__device__ __forceinline__ unsigned long long now_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__global__ void __launch_bounds__(kPassThreads) fmc_pass_server_kernel(DevSystem S, const PassMailbox* mb,
                                                                       PassServerFlags* fl, int* host_words,
                                                                       PassScratch W, long long seq0,
                                                                       long long idle_ns) {
  extern __shared__ double2 sm_tab[];
  __shared__ double red[32 * 2];
  __shared__ double comb[kPassThreads];
  __shared__ bool am_last;
  __shared__ long long s_cmd;
  __shared__ PassArgsT<kSmallPassSites> A;
  __shared__ GuestView G;
  __shared__ const double2* s_sk;
  __shared__ double2* s_sk_new;
  const int tid = threadIdx.x;
  const bool leader = blockIdx.x == 0;
  long long seq = seq0;
  for (;;) {
    if (tid == 0) {
      // block 0 polls the mailbox in host memory, the other blocks block 0's flag in device memory
      const volatile long long* cmd = &mb->cmd;
      const volatile unsigned long long* go = &fl->go;
      const unsigned long long limit = (unsigned long long)(leader ? idle_ns : 64 * idle_ns);
      const unsigned long long t0 = now_ns();
      long long c = -1;
      for (;;) {
        c = leader ? *cmd : (long long)*go;
        if (c > seq) break;
        if (leader ? *(const volatile int*)&mb->quit != 0 : *(volatile int*)&fl->stop != 0) {
          c = -1;
          break;
        }
        if (now_ns() - t0 >= limit) {
          if (!leader) atomicExch(host_words + 1, 1);
          c = -1;
          break;
        }
        __nanosleep(leader ? 64 : 32);
      }
      if (c > seq) {
        // the previous pass's guest-site update is written before this pass reads the sites
        const unsigned long long t1 = now_ns();
        bool late = false;
        while (*(volatile unsigned long long*)&fl->done < (unsigned long long)(c - 1)) {
          if (now_ns() - t1 >= kDoneNs) {
            late = true;
            break;
          }
          __nanosleep(32);
        }
        if (late) {
          atomicExch(host_words + 1, 2);
          c = -1;
        }
      }
      if (c < 0 && leader) {
        *(volatile int*)&fl->stop = 1;
        __threadfence();
      }
      s_cmd = c;
    }
    __syncthreads();
    const long long c = s_cmd;
    if (c < 0) break;
    // the pass into shared memory: block 0 from the mailbox (host memory), which it then copies
    // to device memory for the others; the others from there
    {
      const volatile unsigned long long* src =
          reinterpret_cast<const volatile unsigned long long*>(leader ? (const void*)&mb->A : (const void*)&fl->A);
      unsigned long long* dst = reinterpret_cast<unsigned long long*>(&A);
      for (int i = tid; i < (int)(sizeof(A) / 8); i += blockDim.x) dst[i] = src[i];
      const volatile unsigned long long* gs =
          reinterpret_cast<const volatile unsigned long long*>(leader ? (const void*)&mb->G : (const void*)&fl->G);
      unsigned long long* gd = reinterpret_cast<unsigned long long*>(&G);
      for (int i = tid; i < (int)(sizeof(G) / 8); i += blockDim.x) gd[i] = gs[i];
      if (tid == 0) {
        s_sk = leader ? *(const double2* const volatile*)&mb->sk : *(const double2* const volatile*)&fl->sk;
        s_sk_new = leader ? *(double2* const volatile*)&mb->sk_new : *(double2* const volatile*)&fl->sk_new;
      }
    }
    __syncthreads();
    if (leader) {
      unsigned long long* dA = reinterpret_cast<unsigned long long*>(&fl->A);
      const unsigned long long* sA = reinterpret_cast<const unsigned long long*>(&A);
      for (int i = tid; i < (int)(sizeof(A) / 8); i += blockDim.x) dA[i] = sA[i];
      unsigned long long* dG = reinterpret_cast<unsigned long long*>(&fl->G);
      const unsigned long long* sG = reinterpret_cast<const unsigned long long*>(&G);
      for (int i = tid; i < (int)(sizeof(G) / 8); i += blockDim.x) dG[i] = sG[i];
      if (tid == 0) {
        fl->sk = s_sk;
        fl->sk_new = s_sk_new;
      }
      __threadfence();
      __syncthreads();
      if (tid == 0) *(volatile unsigned long long*)&fl->go = (unsigned long long)c;
    }
    const bool last = pass_block(S, G, A, s_sk, s_sk_new, W, (int)blockIdx.x, (int)gridDim.x, sm_tab, red, comb,
                                 am_last);
    if (last) {
      __syncthreads();  // the update is written by every thread of this block
      if (tid == 0) {
        __threadfence();
        *(volatile unsigned long long*)&fl->done = (unsigned long long)c;
      }
    }
    seq = c;
    __syncthreads();
  }
  // the last block to end tells the host
  if (tid == 0) {
    __threadfence();
    const unsigned n = atomicAdd(&fl->exit_count, 1u);
    if (n == gridDim.x - 1) {
      __threadfence_system();
      *(volatile int*)host_words = 1;
    }
  }
}

int pass_server_blocks(const DevSystem& S) { return pass_recip_blocks(S) + kServerBlocksExtra; }

cudaError_t launch_pass_server(const DevSystem& S, PassMailbox* mb, PassServerFlags* fl, int* host_words,
                               const PassScratch& W, long long seq0, long long idle_ns, cudaStream_t st) {
  static_assert(sizeof(PassArgsT<kSmallPassSites>) % 8 == 0 && sizeof(GuestView) % 8 == 0, "word copies");
  const int grid = pass_server_blocks(S);
  const int smem = pass_smem_bytes(S, kSmallPassSites);
  void* args[] = {(void*)&S, (void*)&mb, (void*)&fl, (void*)&host_words, (void*)&W, (void*)&seq0, (void*)&idle_ns};
  return cudaLaunchCooperativeKernel((const void*)fmc_pass_server_kernel, grid, kPassThreads, args, smem, st);
}

int pass_smem_bytes(const DevSystem& S, int nsite) {
  return nsite * ((S.kmax[0] + 1) + (S.kmax[1] + 1) + (S.kmax[2] + 1)) * (int)sizeof(double2);
}

int pass_recip_blocks(const DevSystem& S) { return (S.K + kPassThreads - 1) / kPassThreads; }

cudaError_t launch_pass(const DevSystem& S, const GuestView& G, const PassArgs& A, const double2* sk, double2* sk_new,
                        const PassScratch& W, cudaStream_t st) {
  int nsite = A.nold + A.nnew;
  int smem = A.nbk > 0 ? pass_smem_bytes(S, nsite) : 0;
  int grid = A.nbk + (A.do_real ? nsite : 0);
  if (grid == 0) return A.pc.op ? cudaErrorInvalidValue : cudaSuccess;  // a pending update needs a block
  if (nsite <= kSmallPassSites) {
    // the common case (molecules of up to 8 sites): a parameter block of ~1.3 KB instead of ~4 KB
    PassArgsT<kSmallPassSites> B;
    std::memcpy(&B, &A, offsetof(PassArgs, x));
    for (int i = 0; i < nsite; i++) {
      B.x[i] = A.x[i];
      B.y[i] = A.y[i];
      B.z[i] = A.z[i];
      B.q[i] = A.q[i];
      B.type[i] = A.type[i];
    }
    B.pc = A.pc;
    fmc_pass_kernel<kSmallPassSites><<<grid, kPassThreads, smem, st>>>(S, G, B, sk, sk_new, W);
  } else {
    fmc_pass_kernel<kMaxPassSites><<<grid, kPassThreads, smem, st>>>(S, G, A, sk, sk_new, W);
  }
  return cudaGetLastError();
}

cudaError_t configure_kernels() {
  cudaError_t e = cudaFuncSetAttribute(fmc_pass_kernel<kSmallPassSites>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       200 * 1024);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(fmc_pass_server_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(fmc_pass_kernel<kMaxPassSites>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  return e;
}


// ------------------------------------------------------------------------------ commit
__global__ void fmc_commit_kernel(int K, double2* sk, const double2* __restrict__ sk_new, CommitArgs C,
                                  double4* site, int* type) {
  if ((int)blockIdx.x < (int)gridDim.x - 1) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < K; k += (gridDim.x - 1) * blockDim.x) sk[k] = sk_new[k];
    return;
  }
  // last block: guest-site segment update
  const int tid = threadIdx.x;
  if (C.op == kDelete) {
    // remove [lo, lo+ns) and shift the rest of the segment down, preserving order
    const int ns = C.ns;
    for (int base = C.lo; base < C.seg_end - ns; base += blockDim.x) {
      int i = base + tid;
      double4 a;
      int t = 0;
      bool act = i < C.seg_end - ns;
      if (act) {
        a = site[i + ns];
        t = type[i + ns];
      }
      __syncthreads();
      if (act) {
        site[i] = a;
        type[i] = t;
      }
      __syncthreads();
    }
  } else if (tid < C.ns) {
    // insert writes at the segment end, displace overwrites the molecule
    site[C.lo + tid] = make_double4(C.x[tid], C.y[tid], C.z[tid], C.q[tid]);
    type[C.lo + tid] = C.type[tid];
  }
}

cudaError_t launch_commit(int K, double2* sk, const double2* sk_new, const CommitArgs& C, double4* site, int* type,
                          cudaStream_t st) {
  int nb = (K + 255) / 256;
  if (nb > 64) nb = 64;
  fmc_commit_kernel<<<nb + 1, 256, 0, st>>>(K, sk, sk_new, C, site, type);
  return cudaGetLastError();
}

// ------------------------------------------------------------------------------ full S(k)
// partial[c*K + k] = sum over the atoms of chunk c (in order) of q e^{i k.r}
constexpr int kRecipThreads = 128;

__global__ void __launch_bounds__(kRecipThreads) fmc_recip_partial_kernel(DevSystem S, const double4* __restrict__ atoms,
                                                                          int natoms, int chunk, double2* partial) {
  extern __shared__ double2 sm_tab[];
  __shared__ double sq[256];
  const int k1 = S.kmax[0], k2 = S.kmax[1], k3 = S.kmax[2];
  const int stride = (k1 + 1) + (k2 + 1) + (k3 + 1);
  const int c = blockIdx.y, a0 = c * chunk;
  const int na = min(chunk, natoms - a0);
  for (int w = threadIdx.x; w < na * 3; w += blockDim.x) {
    int s = w / 3, ax = w % 3;
    double4 a = atoms[a0 + s];
    double f[3];
    frac_coords(S.cell, a.x, a.y, a.z, f);
    double2* t = sm_tab + s * stride + (ax == 0 ? 0 : (ax == 1 ? k1 + 1 : k1 + k2 + 2));
    axis_phases(f[ax], S.kmax[ax], t);
    if (ax == 0) sq[s] = a.w;
  }
  __syncthreads();
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= S.K) return;
  int l, m, n;
  kunpack(S.kpack[k], l, m, n);
  int am = m < 0 ? -m : m, an = n < 0 ? -n : n;
  double2 acc = make_double2(0.0, 0.0);
  for (int s = 0; s < na; s++) {
    const double2* t = sm_tab + s * stride;
    double2 e1 = t[l], e2 = t[k1 + 1 + am], e3 = t[k1 + k2 + 2 + an];
    double2 cc = m >= 0 ? cmul(e1, e2) : cmulc(e1, e2);
    cc = n >= 0 ? cmul(cc, e3) : cmulc(cc, e3);
    acc.x += sq[s] * cc.x;
    acc.y += sq[s] * cc.y;
  }
  partial[(size_t)c * S.K + k] = acc;
}

// S[k] = sum_c partial[c][k]; energy sum akk |S|^2 per block into part[]
__global__ void fmc_recip_reduce_kernel(DevSystem S, const double2* __restrict__ partial, int nchunk, double2* sk,
                                        double* part) {
  __shared__ double red[32];
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  double v[1] = {0.0};
  if (k < S.K) {
    double2 s = make_double2(0.0, 0.0);
    for (int c = 0; c < nchunk; c++) {
      double2 p = partial[(size_t)c * S.K + k];
      s.x += p.x;
      s.y += p.y;
    }
    sk[k] = s;
    v[0] = S.akk[k] * (s.x * s.x + s.y * s.y);
  }
  block_sum<1>(v, red);
  if (threadIdx.x == 0) part[blockIdx.x] = v[0];
}

int recip_chunk(const DevSystem& S) {
  int stride = (S.kmax[0] + 1) + (S.kmax[1] + 1) + (S.kmax[2] + 1);
  int c = (40 * 1024) / (stride * (int)sizeof(double2));  // + 2 KB static charges < 48 KB
  if (c > 256) c = 256;
  return c < 1 ? 1 : c;
}

size_t recip_scratch_doubles(const DevSystem& S, int natoms) {
  int chunk = recip_chunk(S);
  int nchunk = (natoms + chunk - 1) / chunk;
  return (size_t)nchunk * S.K * 2 + 8;
}

int recip_nparts(const DevSystem& S) { return (S.K + 255) / 256; }

cudaError_t launch_recip_full(const DevSystem& S, const double4* atoms, int natoms, double2* sk, double* scratch,
                              double* parts, cudaStream_t st) {
  int chunk = recip_chunk(S);
  int nchunk = (natoms + chunk - 1) / chunk;
  if (nchunk == 0) {
    cudaMemsetAsync(sk, 0, sizeof(double2) * S.K, st);
    return cudaMemsetAsync(parts, 0, sizeof(double) * recip_nparts(S), st);
  }
  int stride = (S.kmax[0] + 1) + (S.kmax[1] + 1) + (S.kmax[2] + 1);
  double2* partial = reinterpret_cast<double2*>(scratch);
  dim3 g((S.K + kRecipThreads - 1) / kRecipThreads, nchunk);
  fmc_recip_partial_kernel<<<g, kRecipThreads, chunk * stride * sizeof(double2), st>>>(S, atoms, natoms, chunk,
                                                                                      partial);
  fmc_recip_reduce_kernel<<<recip_nparts(S), 256, 0, st>>>(S, partial, nchunk, sk, parts);
  return cudaGetLastError();
}

cudaError_t configure_recip_kernels() {
  return cudaFuncSetAttribute(fmc_recip_partial_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 64 * 1024);
}

double recip_energy_from_parts(const DevSystem& S, const double* host_parts) {
  double r = 0.0;
  for (int b = 0; b < recip_nparts(S); b++) r += host_parts[b];
  return S.recip_pref * r;
}

// ------------------------------------------------------------------------------ single point
// For entry b: site i = sites[b]; out[4*b + {0,1,2,3}] = {coulomb vs framework, vdw vs
// framework, coulomb vs other guests, vdw vs other guests}; own molecule = [lo[b], hi[b]).
__global__ void fmc_sp_kernel(DevSystem S, GuestView G, const int* __restrict__ sites, const int* __restrict__ lo,
                              const int* __restrict__ hi, double* out) {
  __shared__ double red[32 * 4];
  const int b = blockIdx.x, i = sites[b];
  double4 a = G.site[i];
  double v[4] = {0.0, 0.0, 0.0, 0.0};
  PendingCommit none;
  none.op = 0;
  none.seg = -1;
  none.lo = none.ns = none.seg_end = 0;
  site_partial(S, G, none, a.x, a.y, a.z, a.w, G.type[i], lo[b], hi[b], threadIdx.x, blockDim.x, v[0], v[1], v[2],
               v[3]);
  block_sum<4>(v, red);
  if (threadIdx.x == 0)
    for (int k = 0; k < 4; k++) out[4 * b + k] = v[k];
}

cudaError_t launch_single_point_rs(const DevSystem& S, const GuestView& G, int nsites, const int* sites, const int* lo,
                                   const int* hi, double* out, cudaStream_t st) {
  if (nsites > 0) fmc_sp_kernel<<<nsites, 256, 0, st>>>(S, G, sites, lo, hi, out);
  return cudaGetLastError();
}

// ------------------------------------------------------------------------------ voxel lists
// Every framework atom whose true minimum-image distance to a voxel's centre is below
// sqrt(lim2) (rcut + the voxel's circumradius), in ascending atom order.
__device__ __forceinline__ double true_dist2_dev(const CellGeom& c, double dx, double dy, double dz) {
  if (c.imcon == 4 || c.imcon == 5 || c.imcon == 7) return shifted_lattice_dist2(c, dx, dy, dz);
  if (c.imcon == 6) return slab_dist2(c, dx, dy, dz);
  min_image(c, dx, dy, dz);
  double best = dx * dx + dy * dy + dz * dz;
  if (c.imcon == 3) {
    for (int i = -1; i <= 1; i++)
      for (int j = -1; j <= 1; j++)
        for (int k = -1; k <= 1; k++) {
          double x = dx + i * c.h[0] + j * c.h[3] + k * c.h[6];
          double y = dy + i * c.h[1] + j * c.h[4] + k * c.h[7];
          double z = dz + i * c.h[2] + j * c.h[5] + k * c.h[8];
          best = fmin(best, x * x + y * y + z * z);
        }
  }
  return best;
}

__device__ __forceinline__ void voxel_centre(const CellGeom& c, int v, int n0, int n1, int n2, double* p) {
  int a = v / (n1 * n2), b = (v / n2) % n1, cc = v % n2;
  double fa = (a + 0.5) / n0, fb = (b + 0.5) / n1, fc = (cc + 0.5) / n2;
  if (c.imcon == 6) {  // slab: in-plane cell, z layers from zlo
    p[0] = fa * c.h[0] + fb * c.h[3];
    p[1] = fa * c.h[1] + fb * c.h[4];
    p[2] = c.zlo + (cc + 0.5) * c.dz;
    return;
  }
  p[0] = fa * c.h[0] + fb * c.h[3] + fc * c.h[6];
  p[1] = fa * c.h[1] + fb * c.h[4] + fc * c.h[7];
  p[2] = fa * c.h[2] + fb * c.h[5] + fc * c.h[8];
}

constexpr int kVoxThreads = 128;

// Voxel prefilter of orthorhombic cells (imcon 1, 2).  code[j] packs atom j's voxel along
// a, b, c (10 bits each); an atom whose voxel lies more than reach voxels away (cyclically)
// along any axis from the list's voxel cannot be within the list radius, so the list kernels
// skip its FP64 distance test.  reach = floor((lim + 0.01 A) / edge + 1.5): half a voxel for
// the atom's place inside its voxel, one for an atom binned into a neighbouring voxel by
// rounding, 0.01 A for rounding of the distance test itself and of the periods.  The lists
// keep exactly the atoms, and the order, of the unfiltered test.
__device__ __forceinline__ int cyclic_gap(int d, int n) {
  d = d < 0 ? -d : d;
  return min(d, n - d);
}

__device__ __forceinline__ bool voxel_near(unsigned cd, int va, int vb, int vc, int n0, int n1, int n2, int3 r) {
  return cyclic_gap(va - (int)(cd & 1023u), n0) <= r.x && cyclic_gap(vb - (int)((cd >> 10) & 1023u), n1) <= r.y &&
         cyclic_gap(vc - (int)(cd >> 20), n2) <= r.z;
}

__global__ void __launch_bounds__(kVoxThreads) fmc_voxel_code_kernel(CellGeom cell, int n0, int n1, int n2,
                                                                     const double4* __restrict__ fw, int nf,
                                                                     unsigned* __restrict__ code) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= nf) return;
  const double4 a = fw[j];
  const double x[3] = {a.x, a.y, a.z};
  const int n[3] = {n0, n1, n2};
  unsigned out = 0;
  for (int k = 0; k < 3; k++) {
    double f = x[k] / cell.h[4 * k];
    f -= floor(f);
    const int i = min(max((int)(f * n[k]), 0), n[k] - 1);
    out |= (unsigned)i << (10 * k);
  }
  code[j] = out;
}

__global__ void __launch_bounds__(kVoxThreads) fmc_voxel_count_kernel(CellGeom cell, int n0, int n1, int n2,
                                                                      const double4* __restrict__ fw, int nf,
                                                                      double lim2, const unsigned* __restrict__ code,
                                                                      int3 reach, int* counts) {
  __shared__ int ws[kVoxThreads / 32];
  double p[3];
  voxel_centre(cell, blockIdx.x, n0, n1, n2, p);
  const int va = blockIdx.x / (n1 * n2), vb = (blockIdx.x / n2) % n1, vc = blockIdx.x % n2;
  int cnt = 0;
  for (int j = threadIdx.x; j < nf; j += blockDim.x) {
    if (code && !voxel_near(code[j], va, vb, vc, n0, n1, n2, reach)) continue;
    double4 a = fw[j];
    if (true_dist2_dev(cell, p[0] - a.x, p[1] - a.y, p[2] - a.z) < lim2) cnt++;
  }
  for (int o = 16; o > 0; o >>= 1) cnt += __shfl_down_sync(0xffffffffu, cnt, o);
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = cnt;
  __syncthreads();
  if (threadIdx.x == 0) {
    int t = 0;
    for (int w = 0; w < kVoxThreads / 32; w++) t += ws[w];
    counts[blockIdx.x] = t;
  }
}

__global__ void __launch_bounds__(kVoxThreads) fmc_voxel_fill_kernel(CellGeom cell, int n0, int n1, int n2,
                                                                     const double4* __restrict__ fw,
                                                                     const int* __restrict__ ftype, int nf, double lim2,
                                                                     const unsigned* __restrict__ code, int3 reach,
                                                                     const int* __restrict__ off, int* atoms,
                                                                     unsigned short* atoms16, double4* xyzq,
                                                                     unsigned char* vtype, long long cap) {
  __shared__ int woff[kVoxThreads / 32 + 1];
  __shared__ int running;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double p[3];
  voxel_centre(cell, blockIdx.x, n0, n1, n2, p);
  const int va = blockIdx.x / (n1 * n2), vb = (blockIdx.x / n2) % n1, vc = blockIdx.x % n2;
  if (threadIdx.x == 0) running = 0;
  const int base = off[blockIdx.x];
  __syncthreads();
  for (int chunk = 0; chunk < nf; chunk += blockDim.x) {
    int j = chunk + threadIdx.x;
    bool flag = false;
    double4 a = make_double4(0, 0, 0, 0);
    if (j < nf && (!code || voxel_near(code[j], va, vb, vc, n0, n1, n2, reach))) {
      a = fw[j];
      flag = true_dist2_dev(cell, p[0] - a.x, p[1] - a.y, p[2] - a.z) < lim2;
    }
    unsigned mask = __ballot_sync(0xffffffffu, flag);
    if (lane == 0) woff[warp + 1] = __popc(mask);
    __syncthreads();
    if (threadIdx.x == 0) {
      woff[0] = 0;
      for (int w = 1; w <= kVoxThreads / 32; w++) woff[w] += woff[w - 1];
    }
    __syncthreads();
    if (flag) {
      int pos = base + running + woff[warp] + __popc(mask & ((1u << lane) - 1u));
      if (pos < cap) {  // beyond the capacity: the caller compares off[nv] with cap and rebuilds
        if (atoms) atoms[pos] = j;
        if (atoms16) atoms16[pos] = (unsigned short)j;
        xyzq[pos] = a;
        vtype[pos] = (unsigned char)ftype[j];
      }
    }
    __syncthreads();
    if (threadIdx.x == 0) running += woff[kVoxThreads / 32];
    __syncthreads();
  }
}

namespace {
int3 voxel_reach(const CellGeom& cell, const int* nvox, double lim2) {
  const double lim = std::sqrt(lim2) + 0.01;
  int r[3];
  for (int a = 0; a < 3; a++) r[a] = (int)std::floor(lim / (cell.h[4 * a] / nvox[a]) + 1.5);
  return make_int3(r[0], r[1], r[2]);
}
}  // namespace

bool voxel_prefilter_applies(const CellGeom& cell, const int* nvox) {
  if (cell.imcon != 1 && cell.imcon != 2) return false;
  for (int a = 0; a < 3; a++)
    if (nvox[a] < 1 || nvox[a] > 1023 || !(cell.h[4 * a] > 0.0)) return false;
  return true;
}

cudaError_t launch_voxel_codes(const CellGeom& cell, const int* nvox, const double4* fw, int nf, unsigned* code,
                               cudaStream_t st) {
  if (nf > 0)
    fmc_voxel_code_kernel<<<(nf + kVoxThreads - 1) / kVoxThreads, kVoxThreads, 0, st>>>(cell, nvox[0], nvox[1],
                                                                                       nvox[2], fw, nf, code);
  return cudaGetLastError();
}

cudaError_t launch_voxel_count(const CellGeom& cell, const int* nvox, const double4* fw, int nf, double lim2,
                               const unsigned* code, int* counts, cudaStream_t st) {
  int nv = nvox[0] * nvox[1] * nvox[2];
  if (code && !voxel_prefilter_applies(cell, nvox)) code = nullptr;
  const int3 r = code ? voxel_reach(cell, nvox, lim2) : make_int3(0, 0, 0);
  fmc_voxel_count_kernel<<<nv, kVoxThreads, 0, st>>>(cell, nvox[0], nvox[1], nvox[2], fw, nf, lim2, code, r, counts);
  return cudaGetLastError();
}

cudaError_t launch_voxel_fill(const CellGeom& cell, const int* nvox, const double4* fw, const int* ftype, int nf,
                              double lim2, const unsigned* code, const int* off, int* atoms, unsigned short* atoms16,
                              double4* xyzq, unsigned char* vtype, long long cap, cudaStream_t st) {
  int nv = nvox[0] * nvox[1] * nvox[2];
  if (code && !voxel_prefilter_applies(cell, nvox)) code = nullptr;
  const int3 r = code ? voxel_reach(cell, nvox, lim2) : make_int3(0, 0, 0);
  fmc_voxel_fill_kernel<<<nv, kVoxThreads, 0, st>>>(cell, nvox[0], nvox[1], nvox[2], fw, ftype, nf, lim2, code, r,
                                                    off, atoms, atoms16, xyzq, vtype, cap);
  return cudaGetLastError();
}

namespace {
constexpr int kScanThreads = 1024;

// Exclusive prefix sum of n counts into off[0..n] (off[n] = total) by one CTA: each thread sums
// a contiguous chunk, the chunk sums are scanned across the block, then each thread writes its
// chunk's offsets.
__global__ void __launch_bounds__(kScanThreads) fmc_exclusive_scan_kernel(const int* __restrict__ counts, int n,
                                                                          int* __restrict__ off) {
  __shared__ int wsum[kScanThreads / 32];
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const int chunk = (n + kScanThreads - 1) / kScanThreads;
  const int lo = min(n, t * chunk), hi = min(n, lo + chunk);
  int sum = 0;
  for (int i = lo; i < hi; i++) sum += counts[i];
  int incl = sum;
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) wsum[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    int w = wsum[lane];
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    wsum[lane] = w;
  }
  __syncthreads();
  int run = incl - sum + (warp ? wsum[warp - 1] : 0);
  for (int i = lo; i < hi; i++) {
    off[i] = run;
    run += counts[i];
  }
  if (t == kScanThreads - 1) off[n] = wsum[kScanThreads / 32 - 1];
}
}  // namespace

cudaError_t launch_exclusive_scan(const int* counts, int n, int* off, cudaStream_t st) {
  fmc_exclusive_scan_kernel<<<1, kScanThreads, 0, st>>>(counts, n, off);
  return cudaGetLastError();
}

}  // namespace fmc
