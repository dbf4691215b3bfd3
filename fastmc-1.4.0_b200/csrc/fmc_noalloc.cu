// Reciprocal-space trial pass for callers that cannot allocate GPU memory.
//
// Some programs that want this energy routine are not allowed to call cudaMalloc: a plug-in
// living inside a host application whose device memory is owned by that application's own
// pool, a solver embedded in a runtime that forbids foreign allocations on its devices, or a
// time-critical loop where an allocation could block or fragment memory.  Such a caller
// already owns every input and output buffer on the device; the only memory this routine
// needs beyond them is a small scratch area, and here that scratch is a fixed array compiled
// into the library image (every GPU that loads the library holds it until the process exits).
//
// Scratch: fmc_noalloc_scratch below -- one energy partial per block of 256 k-vectors (at most
// kNoAllocMaxK / 256 blocks) followed by the last-block ticket.  Every call on a device uses
// the same array and leaves its contents behind; the ticket is cleared before each launch.
// Two calls that overlap on the same GPU (two streams, or two host threads) race on it.
//
// Set-up: the first call on a device (with that device current) looks up the array's device
// address with cudaGetSymbolAddress and caches it; make that first call before any stream
// capture begins.
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>
#include <string>

#include "../../include/fastmc_b200.h"
#include "fmc_device.cuh"

namespace fmc {
void set_last_error(const std::string& msg);  // fmc_api.cu
}

namespace {

constexpr int kNoAllocThreads = 256;
constexpr int kNoAllocMaxK = 32768;
constexpr int kNoAllocMaxBlocks = kNoAllocMaxK / kNoAllocThreads;
constexpr int kNoAllocMaxSites = fmc::kMaxPassSites;
constexpr int kNoAllocMaxDevices = 64;

}  // namespace

// File-scope scratch of the no-allocation pass: block partials, then the ticket.
static __device__ __align__(256) double fmc_noalloc_scratch[kNoAllocMaxBlocks + 2];

namespace {

struct NoAllocPass {
  fmc::CellGeom cell;  // only rh (the inverse cell) is read
  int K, kmax[3], move, nold, nnew, nbk;
  double recip_pref, engsic;
  double x[kNoAllocMaxSites], y[kNoAllocMaxSites], z[kNoAllocMaxSites], q[kNoAllocMaxSites];
};

__global__ void __launch_bounds__(kNoAllocThreads)
    fmc_recip_pass_noalloc_kernel(NoAllocPass P, const int* __restrict__ lmn, const double* __restrict__ akk,
                                  const double* __restrict__ sk, double* sk_new, double* engcpe, double* scratch) {
  using namespace fmc;
  extern __shared__ double2 tab[];
  __shared__ double red[32];
  __shared__ bool am_last;
  const int nsite = P.nold + P.nnew, tid = threadIdx.x;
  const int k1 = P.kmax[0], k2 = P.kmax[1], k3 = P.kmax[2];
  const int stride = (k1 + 1) + (k2 + 1) + (k3 + 1);
  for (int w = tid; w < nsite * 3; w += blockDim.x) {
    int s = w / 3, ax = w % 3;
    double f[3];
    frac_coords(P.cell, P.x[s], P.y[s], P.z[s], f);
    axis_phases(f[ax], P.kmax[ax], tab + s * stride + (ax == 0 ? 0 : (ax == 1 ? k1 + 1 : k1 + k2 + 2)));
  }
  __syncthreads();
  double v[1] = {0.0};
  int k = blockIdx.x * blockDim.x + tid;
  int l = 0, m = 0, n = 0;
  if (k < P.K) {
    l = lmn[3 * k];
    m = lmn[3 * k + 1];
    n = lmn[3 * k + 2];
  }
  int am = m < 0 ? -m : m, an = n < 0 ? -n : n;
  // a k-vector outside the kmax the caller declared would index past the phase tables: its
  // S_new is S and its energy term NaN, so the pass energy comes back NaN
  if (k < P.K && (l < 0 || l > k1 || am > k2 || an > k3)) {
    sk_new[2 * k] = sk[2 * k];
    sk_new[2 * k + 1] = sk[2 * k + 1];
    v[0] = __longlong_as_double(0x7ff8000000000000LL);
  } else if (k < P.K) {
    double2 aold = make_double2(0.0, 0.0), anew = make_double2(0.0, 0.0);
    for (int s = 0; s < nsite; s++) {
      const double2* t = tab + s * stride;
      double2 c = m >= 0 ? cmul(t[l], t[k1 + 1 + am]) : cmulc(t[l], t[k1 + 1 + am]);
      c = n >= 0 ? cmul(c, t[k1 + k2 + 2 + an]) : cmulc(c, t[k1 + k2 + 2 + an]);
      if (s < P.nold) {
        aold.x += P.q[s] * c.x;
        aold.y += P.q[s] * c.y;
      } else {
        anew.x += P.q[s] * c.x;
        anew.y += P.q[s] * c.y;
      }
    }
    double2 so = make_double2(sk[2 * k], sk[2 * k + 1]), sn;
    if (P.move == kInsert)
      sn = make_double2(anew.x + so.x, anew.y + so.y);
    else if (P.move == kDelete)
      sn = make_double2(so.x - aold.x, so.y - aold.y);
    else
      sn = make_double2((so.x - aold.x) + anew.x, (so.y - aold.y) + anew.y);
    sk_new[2 * k] = sn.x;
    sk_new[2 * k + 1] = sn.y;
    v[0] = akk[k] * (sn.x * sn.x + sn.y * sn.y - so.x * so.x - so.y * so.y);
  }
  block_sum<1>(v, red);
  unsigned* ticket = reinterpret_cast<unsigned*>(scratch + kNoAllocMaxBlocks);
  if (tid == 0) {
    scratch[blockIdx.x] = v[0];
    __threadfence();
    am_last = atomicAdd(ticket, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (am_last && tid == 0) {
    __threadfence();
    double r = 0.0;
    for (int b = 0; b < (int)gridDim.x; b++) r += ((volatile double*)scratch)[b];
    double e = P.recip_pref * r;
    if (P.move == kInsert) e = e + P.engsic;
    if (P.move == kDelete) e = e - P.engsic;
    *engcpe = e;
    *ticket = 0u;
  }
}

std::mutex g_mu;
double* g_scratch[kNoAllocMaxDevices] = {nullptr};

int reject(int code, const std::string& msg) {
  fmc::set_last_error(msg);  // reported by fmc_last_error()
  return code;
}

// Device address of the scratch array on the current device (looked up once per device).
int scratch_on_current_device(double** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return reject(-100 - (int)e, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= kNoAllocMaxDevices) return reject(-1, "device ordinal beyond the supported range");
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_scratch[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, fmc_noalloc_scratch);
    if (e != cudaSuccess)
      return reject(-100 - (int)e, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    g_scratch[dev] = static_cast<double*>(p);
  }
  *out = g_scratch[dev];
  return 0;
}

void invert_cell(const double* a, double* b) {
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
  double r = d != 0.0 ? 1.0 / d : 0.0;
  for (int i = 0; i < 9; i++) b[i] = r * b[i];
}

}  // namespace

extern "C" {

int fmc_ewald1_guest_noalloc(int K, const int* kmax, const double* cell, const int* d_lmn, const double* d_akk,
                             const double* d_sk, int move, int nold, int nnew, const double* sites,
                             double recip_pref, double engsic, double* d_sk_new, double* d_engcpe, void* stream) {
  if (!kmax || !cell || !d_lmn || !d_akk || !d_sk || !sites || !d_sk_new || !d_engcpe)
    return reject(-1, "null argument");
  if (K < 1 || K > kNoAllocMaxK)
    return reject(-7, "K = " + std::to_string(K) + " k-vectors is beyond the no-allocation maximum of " +
                          std::to_string(kNoAllocMaxK));
  if (nold < 0 || nnew < 0 || nold + nnew < 1 || nold + nnew > kNoAllocMaxSites)
    return reject(-7, "site count " + std::to_string(nold + nnew) + " is outside 1.." +
                          std::to_string(kNoAllocMaxSites));
  if (!((move == FMC_INSERT && nold == 0) || (move == FMC_DELETE && nnew == 0) || move == FMC_DISPLACE))
    return reject(-1, "move code does not match the old/new site counts");
  for (int a = 0; a < 3; a++)
    if (kmax[a] < 0 || kmax[a] > 127) return reject(-7, "kmax beyond 127");
  double* scratch = nullptr;
  int rc = scratch_on_current_device(&scratch);
  if (rc) return rc;
  NoAllocPass P;
  std::memset(&P, 0, sizeof(P));
  for (int i = 0; i < 9; i++) P.cell.h[i] = cell[i];
  invert_cell(cell, P.cell.rh);
  P.K = K;
  for (int a = 0; a < 3; a++) P.kmax[a] = kmax[a];
  P.move = move == FMC_INSERT ? fmc::kInsert : (move == FMC_DELETE ? fmc::kDelete : fmc::kDisplace);
  P.nold = nold;
  P.nnew = nnew;
  P.nbk = (K + kNoAllocThreads - 1) / kNoAllocThreads;
  P.recip_pref = recip_pref;
  P.engsic = engsic;
  for (int s = 0; s < nold + nnew; s++) {
    P.x[s] = sites[4 * s];
    P.y[s] = sites[4 * s + 1];
    P.z[s] = sites[4 * s + 2];
    P.q[s] = sites[4 * s + 3];
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  // every check before the first device-side effect: a rejected call leaves the scratch alone
  int smem = (nold + nnew) * ((kmax[0] + 1) + (kmax[1] + 1) + (kmax[2] + 1)) * (int)sizeof(double2);
  if (smem > 200 * 1024) return reject(-7, "sites x (kmax1+kmax2+kmax3+3) phase table exceeds 200 KB of shared memory");
  cudaError_t e = cudaSuccess;
  if (smem > 48 * 1024) {
    e = cudaFuncSetAttribute(fmc_recip_pass_noalloc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return reject(-100 - (int)e, cudaGetErrorString(e));
  }
  // the ticket must start at zero: clear it in stream order before the launch
  e = cudaMemsetAsync(scratch + kNoAllocMaxBlocks, 0, sizeof(double), st);
  if (e != cudaSuccess) return reject(-100 - (int)e, std::string("clearing scratch: ") + cudaGetErrorString(e));
  fmc_recip_pass_noalloc_kernel<<<P.nbk, kNoAllocThreads, smem, st>>>(P, d_lmn, d_akk, d_sk, d_sk_new, d_engcpe,
                                                                      scratch);
  e = cudaGetLastError();
  if (e != cudaSuccess) return reject(-100 - (int)e, std::string("launch: ") + cudaGetErrorString(e));
  return 0;
}

}  // extern "C"
