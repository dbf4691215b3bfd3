// Launch interfaces of the plain-path FP64 kernels (fmc_kernels.cu).
#pragma once
#include <cuda_runtime.h>

#include "fmc_device.cuh"

namespace fmc {

// One trial pass: the sites whose reciprocal and real-space contributions change.
// Sites [0, nold) are the molecule's current positions (removed), sites [nold, nold+nnew)
// the trial positions (added).  insert: nold=0; delete: nnew=0; displace: both, fused.
// Arguments of one trial pass for up to N old + new sites.  The kernel is built for N = 16
// (molecules of up to 8 sites, launched with a small parameter block) and for the reference's
// largest molecules (kMaxPassSites); launch_pass picks the smaller one that holds the trial.
template <int N>
struct PassArgsT {
  int move;           // kInsert / kDelete / kDisplace
  int nbk;            // reciprocal blocks (0: skip the reciprocal part)
  int do_real;        // 1: one real-space block per site
  int nold, nnew;
  int ex_lo, ex_hi;   // guest-site range of the moving molecule (excluded from real space)
  double engsic;      // self-interaction term of the species (ewald.f:87-93)
  double seq;         // copied to result[3] after the energies, for a host that polls (0: none)
  double x[N], y[N], z[N], q[N];
  unsigned char type[N];
  PendingCommit pc;   // an accepted guest-site update this pass reads through and then writes
};
constexpr int kSmallPassSites = 16;
using PassArgs = PassArgsT<kMaxPassSites>;

// Scratch of one pass launch (global memory beyond inputs and outputs).
struct PassScratch {
  double* recip_part;  // [ceil(K/256)]
  double* site_e;      // [2*kMaxPassSites]
  unsigned* counter;   // last-block ticket, left at zero by the kernel
  double* result;      // {ewld1, ewld2, vdw, seq} in pinned host memory, written by the kernel directly
  double4* gsite;      // the chain's guest sites and types, written by the last block when the
  int* gtype;          // pass carries a pending update (PassArgs::pc)
};

struct CommitArgs {
  int op;       // kInsert / kDelete / kDisplace
  int lo;       // first site index of the molecule (insert: segment end)
  int ns;       // sites per molecule
  int seg_end;  // delete: current end of the species segment
  double x[kMaxGuestSites], y[kMaxGuestSites], z[kMaxGuestSites], q[kMaxGuestSites];
  int type[kMaxGuestSites];
};

// The resident pass kernel (`fmc_pass_server_kernel`): one launch serves the passes of a chain
// while the host keeps posting them.  The host writes a pass into the mailbox (pinned host
// memory) and then its sequence number; every block polls the number, copies the pass into
// shared memory and does its share as the one-launch kernel does; results go to the same pinned
// words.  Block 0 ends the kernel after an idle time (no pass posted) or on `quit`; every wait
// is bounded on the device clock.
struct PassMailbox {
  long long cmd;     // sequence number of the posted pass, written after everything else
  int quit;          // 1: the kernel ends at its next poll
  int pad;
  GuestView G;
  const double2* sk;
  double2* sk_new;
  PassArgsT<kSmallPassSites> A;
};
// Device-side state of the resident kernel (device memory, set by the host before a launch).
// Only block 0 polls the mailbox over PCIe: it copies each pass into `pass` and then raises
// `go`, which the other blocks poll in device memory.
struct PassServerFlags {
  unsigned long long done;  // last pass whose pending guest-site update has been written
  unsigned long long go;    // last pass block 0 has copied into `pass`
  int stop;                 // block 0 ended the kernel: the other blocks end too
  unsigned exit_count;      // blocks that have ended
  GuestView G;
  const double2* sk;
  double2* sk_new;
  PassArgsT<kSmallPassSites> A;
};
// Pinned host words the resident kernel writes: [0] 1 once every block has ended, [1] 0 or the
// reason a wait ran out (1 a block waited too long for block 0, 2 for the previous pass).
constexpr int kServerBlocksExtra = kSmallPassSites;  // site blocks beyond the reciprocal blocks
cudaError_t launch_pass_server(const DevSystem& S, PassMailbox* mb, PassServerFlags* fl, int* host_words,
                               const PassScratch& W, long long seq0, long long idle_ns, cudaStream_t st);
int pass_server_blocks(const DevSystem& S);

int pass_smem_bytes(const DevSystem& S, int nsite);
int pass_recip_blocks(const DevSystem& S);
cudaError_t configure_kernels();  // once per device, before the first launch
cudaError_t configure_recip_kernels();
cudaError_t launch_pass(const DevSystem& S, const GuestView& G, const PassArgs& A, const double2* sk, double2* sk_new,
                        const PassScratch& W, cudaStream_t st);
cudaError_t launch_commit(int K, double2* sk, const double2* sk_new, const CommitArgs& C, double4* site, int* type,
                          cudaStream_t st);
size_t recip_scratch_doubles(const DevSystem& S, int natoms);
int recip_nparts(const DevSystem& S);
// Full S(k) of `natoms` atoms {x,y,z,q} into sk; per-block sums of akk|S|^2 into parts.
cudaError_t launch_recip_full(const DevSystem& S, const double4* atoms, int natoms, double2* sk, double* scratch,
                              double* parts, cudaStream_t st);
double recip_energy_from_parts(const DevSystem& S, const double* host_parts);
cudaError_t launch_single_point_rs(const DevSystem& S, const GuestView& G, int nsites, const int* sites, const int* lo,
                                   const int* hi, double* out, cudaStream_t st);

// Voxel lists: per voxel, the framework atoms within sqrt(lim2) of its centre by true minimum
// image, in ascending atom order.  Orthorhombic cells (voxel_prefilter_applies) can pass
// per-atom voxel codes (launch_voxel_codes, nf words) so that the FP64 test runs only for atoms
// within reach; code = nullptr tests every atom.  Both give the same lists.
bool voxel_prefilter_applies(const CellGeom& cell, const int* nvox);
cudaError_t launch_voxel_codes(const CellGeom& cell, const int* nvox, const double4* fw, int nf, unsigned* code,
                               cudaStream_t st);
cudaError_t launch_voxel_count(const CellGeom& cell, const int* nvox, const double4* fw, int nf, double lim2,
                               const unsigned* code, int* counts, cudaStream_t st);
cudaError_t launch_voxel_fill(const CellGeom& cell, const int* nvox, const double4* fw, const int* ftype, int nf,
                              double lim2, const unsigned* code, const int* off, int* atoms, unsigned short* atoms16,
                              double4* xyzq, unsigned char* vtype, long long cap,
                              cudaStream_t st);  // entries >= cap not written
// off[0..n]: exclusive prefix sum of counts[0..n-1], off[n] the total (one CTA)
cudaError_t launch_exclusive_scan(const int* counts, int n, int* off, cudaStream_t st);

}  // namespace fmc
