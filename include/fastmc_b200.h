/* fastmc_b200.h -- C ABI of the B200 GCMC trial-move energy path.
 *
 * Drop-in boundary for FastMC 1.4.0's energy routines.  Plain C types only: pointers, sizes,
 * int status codes.  Status: 0 = ok; > 0 = the reference's own error code (error.f: 3, 4, 25,
 * 52-55, 75, 95, 380, 410, 2311, 2312); < 0 = this library (-2 directive outside the path,
 * -4 a cell without periodic boundaries (imcon 0), -5 too many species, -6 non-rigid
 * framework, -100-e = CUDA error e).  fmc_last_error() gives the message of the
 * calling thread's last failure.
 *
 * Coordinates are Angstrom, interleaved x,y,z per site; energies follow the reference's
 * internal units (10 J/mol) unless stated as kcal/mol.  Host pointers are caller-owned and
 * only read or written during the call.  One chain handle must not be used by two host threads
 * at once; distinct handles may.
 */
#ifndef FASTMC_B200_H
#define FASTMC_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct fmc_chain fmc_chain;

/* Move-type codes (gcmc.f:753-778): insert, delete, displace (translate+rotate),
 * translate-only, rotate-only. */
#define FMC_INSERT 1
#define FMC_DELETE 2
#define FMC_DISPLACE 3
#define FMC_TRANSLATE 4
#define FMC_ROTATE 5

/* One attempted move of the move loop; energies as in gcmc.f:946,1112,1328 (internal units
 * except estep and energy_after, kcal/mol). */
typedef struct fmc_move_record {
  int32_t step, iguest, mtype, randchoice, accepted, nmols_after, pad0, pad1;
  double ewld1, ewld2, ewld3, vdw, delrc, estep, rande, energy_after;
} fmc_move_record;

int fmc_version(void);
const char* fmc_last_error(void);

/* Reads dir/CONTROL, dir/FIELD and dir/CONFIG (readinputs.f:11-914, utility_pack.f:176-457),
 * builds the tables (erfcgen ewald.f:1; forgen vdw_terms.f:189), uploads the rigid framework,
 * computes the single-point energy (gcmc.f:2518-2710) and S(k) of all atoms (gcmc.f:522), and
 * seeds duni (gcmc.f:2712) with seed[0..3] = the (i,j,k,l) the reference prints.  When CONTROL
 * says `restart` (readinputs.f:604-608) the chain is node 0 of its job and continues from the
 * REVIVE fmc_restart_branch picks beside the deck, as fmc_chain_restart would. */
int fmc_chain_open(const char* dir, const int* seed, int device, fmc_chain** out);
/* fmc_chain_open as node `idnode` (0-based; the reference's MPI rank) of a job run from one deck
 * directory: only a CONTROL `restart` reads it, to pick the node's branch (gcmc.f:353-394). */
int fmc_chain_open_node(const char* dir, const int* seed, int device, int idnode, fmc_chain** out);
/* The branch choice of CONTROL `restart` (gcmc.f:353-394 with revscan, utility_pack.f:1819-1839):
 * prevnodes = the entries of `workdir` whose names contain "branch"; node idnode reads
 * branch{idnode+1}/REVIVE when idnode < prevnodes, else branch{mod(idnode+1, prevnodes)+1}/REVIVE,
 * and starts from the CONFIG when there are no branches or that REVIVE does not exist (revread,
 * utility_pack.f:1855-1860).  Writes the REVIVE's path ("" for the CONFIG) and the node's output
 * directory workdir/branch{idnode+1} (NUL-terminated; either buffer may be NULL with cap 0) and
 * *prevnodes (may be NULL).  Returns 1 when a REVIVE is read, 0 when the node starts from the
 * CONFIG, < 0 for bad arguments, idnode outside 0-98 or a buffer too small.  A batch
 * (fmc_batch_open) numbers the chains of one deck directory 0, 1, ... in order as its nodes. */
int fmc_restart_branch(const char* workdir, int idnode, char* revive_path, int revive_cap, char* outdir,
                       int outdir_cap, int* prevnodes);
/* Passes of up to 8-site molecules run through a resident kernel (no counterpart in the
 * reference): it stays on the GPU while passes keep coming, takes each from pinned host memory
 * and ends after ~20 ms without one; the next pass starts it again.  enable 1 / 0 turns it on /
 * off (off by default), -1 only reports; *launches and *passes count its launches and the passes
 * it served.  Returns 1 if on, 0 if off (it also switches itself off when the GPU cannot hold all
 * its blocks at once). */
int fmc_chain_resident(fmc_chain* c, int enable, long long* launches, long long* passes);
void fmc_chain_close(fmc_chain* c);

/* ---------------------------------------------------------------- system from caller arrays
 * The state the reference keeps in its module arrays once readfield / readconfig / readcontrol
 * have run (utility_pack.f:8-68, vdw_module.f:19-24), handed over by pointer instead of files:
 * a Fortran caller whose in-memory state differs from the decks on disk (a restart remap,
 * gcmc.f:353-418, or a framework it generated) passes c_loc of its own arrays.  Types are
 * 1-based as the reference's ltype; energies of vdW parameters in internal units (10 J/mol, the
 * reference's prmvdw after the FIELD `units` scaling). */
typedef struct fmc_guest_desc {
  const char* name;              /* species name (NUL-terminated; NULL: "guest") */
  int nsite;                     /* sites per molecule (1-50; 16 on the batched path) */
  const char* const* site_name;  /* [nsite] site names, or NULL (the type names) */
  const double* mass;            /* [nsite] */
  const double* charge;          /* [nsite] e */
  const double* tx;              /* [nsite] template, centred on the mass centre (readinputs.f:246-268) */
  const double* ty;
  const double* tz;
  const int* type;               /* [nsite] atom types, 1-based */
  int nmols;                     /* molecules present (framwkxxx rows) */
  const double* xyz;             /* [3*nmols*nsite] x,y,z per site, molecule-major; NULL if nmols = 0 */
  double pressure_pa;            /* partial pressure, Pa (the reference's gstpress) */
  double move_freq[9];           /* move weights: insert, delete, displace, jump, flex, swap, translate,
                                    rotate, multi-jump (gcmc.f:282-331 normalises them) */
  double disp_ratio, tran_ratio; /* target acceptance of displacements / translations (0.5 in CONTROL) */
} fmc_guest_desc;

/* One vdW pair line (define_van_der_waals, vdw_terms.f:1-187): the two atom types, the form
 * (keypot: 1 12-6, 2 lj, 3 n-m, 4 buck, 5 bhm, 6 hbnd, 7 shifted n-m, 8 morse, 9 wca) and its
 * five parameters with energies in internal units.  Pairs without a line get the zero table. */
typedef struct fmc_vdw_desc {
  int type_i, type_j, form;
  double prm[5];
} fmc_vdw_desc;

typedef struct fmc_system_desc {
  int imcon;                       /* 1-7 (imcon 0 has no device path) */
  double cell[9];                  /* cell vectors a, b, c (Angstrom) */
  double alpha;                    /* Ewald alpha (1/Angstrom) */
  int kmax[3];
  double rcut, rvdw, delr;         /* rvdw 0: rcut */
  double engunit;                  /* internal units per FIELD energy unit (kcal/mol: 418.4) */
  int ntypes;                      /* unique atom types */
  const char* const* type_names;   /* [ntypes] names (8 characters), or NULL ("T1", "T2", ...) */
  int nframework;                  /* rigid framework atoms, condensed order */
  const double* fw_xyz;            /* [3*nframework] */
  const double* fw_charge;         /* [nframework] */
  const int* fw_type;              /* [nframework] 1-based */
  const double* fw_mass;           /* [nframework] or NULL (only the probability-cube writer reads it) */
  int nguest;                      /* guest species (1-4) */
  const fmc_guest_desc* guests;    /* [nguest] */
  int nvdw;                        /* vdW pair lines */
  const fmc_vdw_desc* vdw;         /* [nvdw] */
  double temperature;              /* K */
  int eq_steps, prod_steps;        /* CONTROL equilibration / steps (negative: cycles of N+1 moves) */
  int max_guest_atoms;             /* CONTROL `max guest atoms` (0: 3000) */
  int averaging_window;            /* CONTROL `averaging window` (0: 100000) */
  int acceptance_sampling;         /* CONTROL `sampling` (statistics only on accepted moves) */
  double rota_ratio;               /* target acceptance of rotations (0: 0.5) */
  void* owner;                     /* set by fmc_deck_describe for fmc_desc_free; callers leave NULL */
} fmc_system_desc;

/* fmc_chain_open from a descriptor instead of a deck directory (no counterpart in the reference,
 * whose state lives in module arrays): the same tables, single point and S(k).  The arrays are
 * read during the call only. */
int fmc_chain_create(const fmc_system_desc* desc, const int* seed, int device, fmc_chain** out);
/* Host only: read a deck directory into a descriptor whose arrays the library owns (release
 * them with fmc_desc_free).  A caller may change the arrays it points to -- the guests present,
 * say -- before fmc_chain_create. */
int fmc_deck_describe(const char* dir, fmc_system_desc* out);
void fmc_desc_free(fmc_system_desc* desc);
/* sizeof of fmc_system_desc, fmc_guest_desc and fmc_vdw_desc in out[0..2] (binding checks). */
int fmc_desc_sizes(int* out);
/* Host only: the tables a descriptor builds, as fmc_deck_inspect reports them for a deck, plus
 * the vdW tables (vvv[ntables*(mxgrid+1)], table 1 first; NULL to skip, *ntables their count). */
int fmc_desc_inspect(const fmc_system_desc* desc, int* ints, double* dbls, int* lmn, double* akk, double* erc,
                     double* charges, int* K, int* nerc, double* vvv, int* ntables);

/* ints[0..15]: imcon, kmax1, kmax2, kmax3, K (newld), total atoms, guest species, atom types,
 * mxgrid, framework atoms, moves done, voxel count, guest-site capacity, 0, 0, 0.
 * dbls[0..15]: alpha, rcut, delr, volume, engunit, temperature, beta, drewd, dlrpot,
 * spenergy (kcal/mol), dlpeng (kcal/mol), framework recip+self (internal), elrc, energy of
 * species 0 (kcal/mol), volume in m^3, 0. */
int fmc_chain_info(fmc_chain* c, int* ints, double* dbls);

/* ewald1 (ewald.f:368-630): recomputes S(k) over every atom now present and returns the
 * reciprocal + self energy (internal units) and K. */
int fmc_ewald1(fmc_chain* c, double* engcpe, int* newld);

/* ewald1_guest (ewald.f:32-365) for one pass of species `iguest` (0-based) with `natms`
 * sites at xyz.  move: FMC_INSERT, FMC_DELETE, FMC_DISPLACE; pass 1 or 2 for FMC_DISPLACE as
 * in the reference (pass 1 stores the old sites and returns 0; pass 2 returns the energy of
 * the displacement).  S_new stays on the device until fmc_commit. */
int fmc_ewald1_guest(fmc_chain* c, int iguest, int natms, const double* xyz, int move, int pass, double* engcpe);

/* guestlistgen + images + ewald2 + srfrce (utility_pack.f:3113-3177, ewald.f:632-694,
 * vdw_terms.f:398-498): real-space Coulomb and vdW of the sites at xyz against every atom
 * except molecule `mol` (0-based index within the species, -1 for none). */
int fmc_guest_realspace(fmc_chain* c, int iguest, int natms, const double* xyz, int mol, double* ewld2, double* vdw);

/* Accept the last evaluated move: S(k) <- S_new (gcmc.f:971-974) and the species' site
 * arrays updated (insert appends at the end, delete removes molecule `mol` keeping order,
 * displace overwrites molecule `mol`; gcmc.f:966-970, 1134-1138, 1352-1357). */
int fmc_commit(fmc_chain* c, int move, int iguest, int mol, const double* xyz);

/* Reject the last evaluated move: S(k) and the sites stay as they were (the reference skips the
 * commit, gcmc.f:954-1002) and the pending S_new is dropped; the next pass overwrites it.  It
 * touches no device memory and is there so that a caller states either outcome. */
int fmc_reject(fmc_chain* c);

/* The same three calls on separate coordinate arrays, as the reference's module arrays
 * newx/newy/newz hold a trial molecule (ewald1_guest ewald.f:32-365, guestlistgen
 * utility_pack.f:3113-3177, the commit gcmc.f:966-982): x[natms], y[natms], z[natms]. */
int fmc_ewald1_guest_xyz(fmc_chain* c, int iguest, int natms, const double* x, const double* y, const double* z,
                         int move, int pass, double* engcpe);
int fmc_guest_realspace_xyz(fmc_chain* c, int iguest, int natms, const double* x, const double* y, const double* z,
                            int mol, double* ewld2, double* vdw);
int fmc_commit_xyz(fmc_chain* c, int move, int iguest, int mol, const double* x, const double* y, const double* z);

/* Replaces all molecules of species `iguest` (the condense of utility_pack.f:3325), then
 * recomputes S(k).  xyz holds nmol*nsite sites, molecule-major. */
int fmc_set_guests(fmc_chain* c, int iguest, int nmol, const double* xyz);

/* single_point (gcmc.f:2518-2710) of the current state: guest energy and the DL_POLY total,
 * both kcal/mol. */
int fmc_single_point(fmc_chain* c, double* spenergy, double* dlpeng);

/* S(k) (current, or the pending S_new) as separate real/imaginary arrays of K values. */
int fmc_get_sk(fmc_chain* c, int pending, double* re, double* im);
/* k-vector table in the reference's order: lmn[3K] and akk[K]. */
int fmc_kvectors(fmc_chain* c, int* lmn, double* akk);

/* The plain GPU move loop: `nmoves` iterations of gcmc.f:589-1380 on the host with every
 * energy evaluated on the device; trace (nullable) receives one record per move. */
int fmc_run(fmc_chain* c, int nmoves, fmc_move_record* trace);

/* Guest coordinates of species `iguest` (nmol*nsite sites, molecule-major); *nmol and *nsite
 * are set; xyz may be NULL to query the counts. */
int fmc_guest_coords(fmc_chain* c, int iguest, double* xyz, int* nmol, int* nsite);

/* Rolling production statistics of species `iguest` (gcmc.f:1814-1860):
 * out[0..5] = <N>, <E>, <EN>, <N^2>, <E^2>, production moves counted. */
int fmc_stats(fmc_chain* c, int iguest, double* out);

/* ---------------------------------------------------------------- checkpoint / restart
 * REVIVE and REVCON in the reference's formats (revive, utility_pack.f:1772-1817; revread,
 * 1840-1878): REVIVE is Fortran unformatted sequential (4-byte little-endian record markers):
 * production flag, nummols per FIELD molecule type, chainstats(1+14*nguest), natms, x/y/z per
 * molecule type, energy per guest species.  A restart (gcmc.f:353-418) loads the guests,
 * recomputes the single point and sets every species' energy to it, keeps the production flag
 * unless a positive equilibration count follows, restores chainstats and restarts prodcount. */
/* Writes outdir/REVIVE and outdir/REVCON for a deck and a state given on the host (no GPU):
 * nmol[nguest]; guest_xyz = every species' interleaved xyz, species after species. */
int fmc_revive_write_state(const char* deck_dir, const char* outdir, int production, const int* nmol,
                           const double* guest_xyz, const double* chainstats, const double* energy, double eng);
/* Reads a REVIVE against the deck's FIELD; any output may be NULL (nmol first to size guest_xyz). */
int fmc_revive_read(const char* path, const char* deck_dir, int* production, int* nmol, double* guest_xyz,
                    double* chainstats, double* energy, int* natms);
int fmc_chain_write_revive(fmc_chain* c, const char* outdir);  /* replaces revive */
int fmc_chain_restart(fmc_chain* c, const char* revive_path);   /* replaces revread + restart */

/* ---------------------------------------------------------------- pressure equilibration
 * CONTROL `desorb 1`, `adsorb press`, `adsorb guests`, `packing fraction` and `finishment d`
 * make the equilibration adjust the partial pressures every 400 moves (gcmc.f:637-696) until the
 * rate falls under d.  out[ng + 1]: the partial pressures (Pa) the acceptance uses now, then the
 * tolerance still in force (0 once equilibrated). */
int fmc_chain_pressures(fmc_chain* c, double* out);

/* ---------------------------------------------------------------- trajectory files
 * numguests.out (gcmc.f:1937-1951): every nnumg moves (CONTROL `numguests`, else
 * max(1, equilibration / 1000)) one line per species: move, molecules, energy, the move's dE
 * and its insert/delete/displace/jump/flex/swap flags.  his.xyz (hisarchive, gcmc.f:2491-2517):
 * every |nhis| moves (CONTROL `history`; positive: production only) the guest sites before the
 * move.  Mixtures get numguestsNN.out / hisNN.xyz per species.  The plain chain writes both
 * while they are open (NULL closes them); a batched chain's numguests.out is rebuilt from the
 * move trace of its last run (`append` adds to the file). */
int fmc_chain_open_outputs(fmc_chain* c, const char* outdir);

/* ---------------------------------------------------------------- statistics
 * The reference's averaging windows (gcmc.f:1814-1928) run on every production move; the final
 * statistics (gcmc.f:1960-2037) use 5 blocks of the first production samples up to 500,000
 * production moves, the closed windows beyond.  final_stats out[1 + 14 ng]: production moves,
 * then per species <N>, <E>, <EN>, <N^2>, <E^2>, the sixth average, and the errors of N, E, EN,
 * N^2, E^2, Q_st, Cv and the sixth.  window_stats out[2 + 24 ng + ng ng]: avcount, rollcount,
 * the window sums, variances and current means (8 per species), the selectivities.  The report
 * is the reference's per-node block (gcmc.f:2052-2117). */
int fmc_chain_window_stats(fmc_chain* c, double* out);
int fmc_chain_final_stats(fmc_chain* c, double* out);
int fmc_chain_write_report(fmc_chain* c, const char* path);
/* The same report from statistics already at hand (pooled over chains, say), on the host
 * alone: final_stats in the layout above, seltot[ng ng] species-major or NULL. */
int fmc_write_report(const char* deck_dir, const double* final_stats, const double* seltot, const char* path);

/* ---------------------------------------------------------------- probability plots
 * CONTROL `probability` plots (per guest: sites binned, 0 = centre of mass), `grid spacing`,
 * `grid factors`.  Every production move bins each guest molecule's sites into its species'
 * plots by equitable_bin (storeprob, utility_pack.f:496-561, 1880-1990).  dims[4]: plots, then
 * grid cells along a, b, c; out: one plot's na*nb*nc summed weights, c fastest.  The cube
 * writers emit prob_guestGG_prob_PP.cube per plot (writeprob, utility_pack.f:563-648), density
 * per Bohr^3 per production move, nothing before production. */
int fmc_chain_prob(fmc_chain* c, int plot, int* dims, double* out);
/* Host only: one plot's grid written as a cube file for a deck; the atomic number the cube
 * files give a mass (the reference's atmnumber mass windows, utility_pack.f:1992-2237). */
int fmc_write_prob_cube(const char* deck_dir, const char* path, const double* grid, long long steps);
int fmc_atomic_number(double mass);
int fmc_chain_write_prob(fmc_chain* c, const char* outdir);

/* ---------------------------------------------------------------- batched path
 * Many independent chains (isotherm points) advanced by one persistent kernel, one CTA per
 * chain, the whole move loop of gcmc.f:589-1380 on the device (no counterpart in the
 * reference, which runs one chain per MPI rank, gcmc.f:334-417).  Chains are opened from
 * their own CONTROL/FIELD/CONFIG directories (guests the deck preloads included), and chains
 * whose FIELD, CONFIG, cut-offs and Ewald parameters coincide share one device system. */
typedef struct fmc_batch fmc_batch;
int fmc_batch_open(int nchains, const char* const* dirs, const int* seeds, int device, fmc_batch** out);
/* The same with the edge (A, 0.5-8) of the voxels whose neighbour lists the kernel reads
 * (fmc_batch_open uses 2 A): finer voxels mean shorter lists per trial site and more memory. */
int fmc_batch_open_edge(int nchains, const char* const* dirs, const int* seeds, int device, double voxel_edge,
                        fmc_batch** out);
/* Autotuner of the voxel edge: opens a throwaway batch of the same chains for every candidate
 * edge, runs `moves` moves twice and keeps the edge whose second launch was fastest (device ms of
 * each candidate in ms[nedges] when given).  The chains the caller opens afterwards start afresh. */
int fmc_batch_autotune(int nchains, const char* const* dirs, const int* seeds, int device, const double* edges,
                       int nedges, int moves, double* best_edge, float* ms);
void fmc_batch_close(fmc_batch* b);
/* Advances every chain by `moves` trial moves in one launch; trace (nullable) receives
 * nchains*moves records, chain-major; *device_ms is the launch's CUDA-event time.  A chain
 * stops after the move on which its deck's equilibration + production cycles end (the
 * reference's loop test, gcmc.f:594-736); its later records stay as the caller left them. */
int fmc_batch_run(fmc_batch* b, int moves, fmc_move_record* trace, float* device_ms);
/* enable != 0: later runs accumulate SM clock cycles per phase of the move (see
 * fmc_batch_chain_state out[27..31]). */
int fmc_batch_profile(fmc_batch* b, int enable);
/* out[0..39]: status, moves done, gcmccount, nmol[4], energy[4] (kcal/mol), elrc, accepted
 * insertions, accepted deletions, insert attempts, delete attempts, production moves,
 * species-0 <N>,<E>,<EN>,<N^2>,<E^2>, system index, K, framework atoms, T, P(species 0),
 * profiled cycles of: trial set-up, phase tables, energy sums, acceptance, commit, then
 * (thread 0's share) k-space, + real space, move selection, trial generation, then 1 once the
 * chain has finished (out[37..39] 0). */
int fmc_batch_chain_state(fmc_batch* b, int chain, double* out);
/* Load balance of the last run (no counterpart in the reference): out[0..2] = the chain's CTA
 * start and end on the device clock (%globaltimer, ns) and the SM it ran on.  Recorded on every
 * run (two clock reads per CTA); 0 for a chain that has not run. */
int fmc_batch_chain_timing(fmc_batch* b, int chain, long long* out);
/* Tile shapes of the batched kernel (no counterpart in the reference, which evaluates one trial
 * per call): threads per chain, k-vectors per thread per trip of the reciprocal loop
 * (ewald.f:145-331), neighbour candidates per trip of the real-space loop (ewald.f:656-690,
 * vdw_terms.f:455-495).  fmc_batch_tiles fills up to cap entries and returns the count; tile 0
 * is the default.  Tiles of one thread count give bit-identical results.  Phase profiling
 * (fmc_batch_profile) runs tile 0 only. */
int fmc_batch_tiles(int* threads, int* kvec_per_trip, int* cand_per_trip, int cap);
int fmc_batch_set_tile(fmc_batch* b, int tile);
int fmc_batch_get_tile(fmc_batch* b);
/* Times the given tiles on a throwaway batch of the same chains at voxel_edge: warm_moves
 * moves first, then `moves` per launch, each tile launched twice in palindromic order; ms[i]
 * the mean launch time of tiles[i], *best_tile the fastest. */
int fmc_batch_autotune_tiles(int nchains, const char* const* dirs, const int* seeds, int device, double voxel_edge,
                             const int* tiles, int ntiles, int warm_moves, int moves, int* best_tile, float* ms);
int fmc_batch_guest_coords(fmc_batch* b, int chain, int iguest, double* xyz, int* nmol, int* nsite);
/* The neighbour lists of a chain's system as the device built them (guestlistgen's candidate
 * sets, utility_pack.f:3113-3177, precomputed per voxel): nvox[0..2], off[nvox+1] (CSR
 * offsets; NULL to skip), atoms[cap] (0-based framework atom indices, ascending in each voxel;
 * NULL to skip), *n_entries. */
int fmc_batch_voxels(fmc_batch* b, int chain, int* nvox, int* off, int* atoms, long long cap, long long* n_entries);
/* Checkpoint / restart of one chain of a batch (formats as fmc_chain_write_revive).  A restart
 * before the chain's first run matches the reference's restart, which re-seeds duni. */
int fmc_batch_write_revive(fmc_batch* b, int chain, const char* outdir);
int fmc_batch_restart(fmc_batch* b, int chain, const char* revive_path);
/* Probability plots of one chain of a batch (as fmc_chain_prob; the device sums weights in
 * fixed point, 2^-32 units, so the grids do not depend on the order of the adds). */
int fmc_batch_prob(fmc_batch* b, int chain, int plot, int* dims, double* out);
/* Statistics of one chain of a batch (as the fmc_chain_ functions; the stored samples live on
 * the device, 16 MB a species a chain). */
int fmc_batch_window_stats(fmc_batch* b, int chain, double* out);
/* Partial pressures of one chain of a batch (as fmc_chain_pressures). */
int fmc_batch_pressures(fmc_batch* b, int chain, double* out);
/* numguests.out of one chain of a batch (see the trajectory files above). */
int fmc_batch_write_numguests(fmc_batch* b, int chain, const void* trace, int nmoves, const char* outdir,
                              int append);
/* Bytes of one chain's control block (copied host->device and back around every run). */
int fmc_batch_control_block_bytes(void);
/* Bytes of one system's constant block (a serving slot copies it host->device every step). */
int fmc_system_block_bytes(void);
int fmc_batch_final_stats(fmc_batch* b, int chain, double* out);
int fmc_batch_write_report(fmc_batch* b, int chain, const char* path);
int fmc_batch_write_prob(fmc_batch* b, int chain, const char* outdir);

/* ---------------------------------------------------------------- serving
 * Isotherm-point requests (an input-deck directory, a duni seed and a budget) served with
 * continuous batching on one GPU: fmc_server_step admits queued requests into free slots while
 * the device-memory budget allows (mem_budget 0: 80% of the free memory), advances every
 * running request by up to `moves` moves in one persistent launch, and retires finished ones,
 * freeing their slots for the next step.  k_capacity bounds the k-vectors of any request
 * (with guests of up to 4 sites and kmax <= 32 per axis; larger requests are rejected).
 * A request's budget is `moves` trial moves, or with moves = 0 its deck's own equilibration +
 * production cycles (CONTROL `equilibration` / `steps`).  A request starts from the empty
 * framework, or from the guests its deck preloads (FIELD NUMMOLS > 0), or, when CONTROL says
 * `restart`, from the REVIVE fmc_restart_branch picks for node 0 (written by the reference, a
 * plain chain or a batched one); the single point of such a start state is computed on the
 * device at preparation by a chain opened on the deck and closed again. */
typedef struct fmc_server fmc_server;
int fmc_server_open(int slots, int device, long long mem_budget, int k_capacity, fmc_server** out);
void fmc_server_close(fmc_server* s);
int fmc_server_submit(fmc_server* s, const char* dir, const int* seed, long long moves, int* request_id);
/* Neighbour-list voxel edge (A, 1-4; 2 by default) of the slots of requests prepared after the
 * call: coarser voxels mean fewer lists to build at admission and less slot memory, and more
 * candidates per trial site. */
int fmc_server_set_voxel_edge(fmc_server* s, double edge);
/* Host only: a deck's device footprint as a serving slot or batched chain (*bytes, the estimate
 * admission uses) and the algorithmic bytes of one of its moves (*move_cost), for placing
 * chains and requests on GPUs by HBM footprint and load (fastmc_b200.placement). */
int fmc_deck_footprint(const char* dir, double voxel_edge, long long* bytes, double* move_cost);
int fmc_server_cancel(fmc_server* s, int request_id);
/* Checkpoints of served requests (revive, utility_pack.f:1772-1817, for requests instead of MPI
 * ranks): with enable = 1, every request that finishes from then on has its guests copied to the
 * host as its slot is freed (off by default: one small device-to-host copy per retirement);
 * fmc_server_write_revive then writes that final state as REVIVE + REVCON into outdir, in the
 * formats fmc_chain_write_revive writes.  A later request on the same deck with CONTROL `restart`
 * and that REVIVE as branch01/REVIVE resumes from it.  Only finished requests are kept (not
 * cancelled or rejected ones); writing any other request fails. */
int fmc_server_keep_final_state(fmc_server* s, int enable);
int fmc_server_write_revive(fmc_server* s, int request_id, const char* outdir);
/* One step of the pipelined server: queues the next launch of every running request (after the
 * uploads of the requests admitted by the previous step), then completes the launch queued by
 * the previous step -- its finished requests are retired -- and admits queued requests into free
 * slots, set up beside the launch in flight for the launch after it.  So the device runs launch
 * after launch while the host retires and admits.  *active: requests in the completed launch
 * (0 on a step that completed none); *device_ms: its device time; *queued: requests still
 * waiting.  Requests keep stepping while fmc_server_busy reports work. */
int fmc_server_step(fmc_server* s, int moves, int* active, int* queued, float* device_ms);
/* *busy = 1 while a launch is in flight, a request runs or one is queued. */
int fmc_server_busy(fmc_server* s, int* busy);
/* Requests that reached a final state (done, rejected, cancelled) since the last call, oldest
 * first, at most cap: ids[cap], states[cap] and results[cap*32] (the layout of fmc_server_poll)
 * -- one call per step instead of a poll per live request. */
int fmc_server_poll_done(fmc_server* s, int* ids, int* states, double* results, int cap, int* n);
/* *state: 0 queued, 1 running, 2 done, -1 rejected (message in fmc_last_error), -2 cancelled.
 * A running request's results are those of the last completed launch.
 * out[0..31]: moves done, status, nmol[4], energy[4] (kcal/mol), production moves,
 * species-0 <N>,<E>,<EN>,<N^2>,<E^2>, accepted insertions, accepted deletions, 0,
 * K, framework atoms, T, P(species 0), move budget, 1 if the deck's cycles finished,
 * species-1 <N>,<E>,<EN>,<N^2>,<E^2>, gcmccount, 0. */
int fmc_server_poll(fmc_server* s, int request_id, int* state, double* out);
int fmc_server_memory(fmc_server* s, long long* used, long long* budget);
/* out[0..13]: requests admitted, retired, launches, host ms spent admitting (device set-up of
 * new slots, incl. waits), device ms of the launches, ms waited for host preparation with
 * nothing running, worker ms preparing requests (summed over threads), worker threads, trial
 * moves run in all launches, trial moves run in the last step's launch, worker ms parsing
 * decks and building host tables, worker ms enqueueing device slots ahead (the builds run on
 * the workers' streams without the workers waiting), admissions that installed a slot built
 * ahead, admissions built at admission.  Deck parsing and host tables run on worker threads
 * ahead of admission. */
int fmc_server_stats(fmc_server* s, double* out);

/* Launch accounting and timing of the plain path.  enable != 0 turns on CUDA-event timing of
 * every trial-pass kernel on the chain's stream (enable < 0 also clears the counters).
 * out[0..5]: trial-pass launches, commit launches, timed pass launches, total timed pass
 * kernel ms, K, sites scanned per pass (framework voxel-list mean). */
int fmc_chain_profile(fmc_chain* c, int enable, double* out);

/* fmc_run with the run bracketed by CUDA events on the chain's stream: *device_ms receives
 * the elapsed device time of the whole run (host move loop included, as it drives the GPU). */
int fmc_run_timed(fmc_chain* c, int nmoves, fmc_move_record* trace, float* device_ms);

/* Reciprocal-space trial pass that allocates nothing (no counterpart in the reference; its
 * arithmetic is that of fmc_ewald1_guest).  For callers that may not call cudaMalloc -- a
 * plug-in whose device memory belongs to the host application's own pool, or a loop where an
 * allocation must not happen -- and that already hold every buffer on the current device:
 *   d_lmn[3K] (l,m,n per k-vector, order of fmc_kvectors), d_akk[K], d_sk[2K] (Re,Im pairs),
 *   outputs d_sk_new[2K] and d_engcpe[1] (the pass energy, internal units, as ewald1_guest);
 *   host arrays kmax[3], cell[9] (cell vectors a,b,c), sites[4*(nold+nnew)] (x,y,z,q; the nold
 *   old sites first); recip_pref = 2*(2 pi/V)*r4pie0, engsic the species' self term.
 * move: FMC_INSERT (nold = 0), FMC_DELETE (nnew = 0) or FMC_DISPLACE (both, one fused pass).
 * Every k-vector of d_lmn must lie inside kmax (|l|,|m|,|n| <= kmax[0..2]); one outside makes the
 * pass energy NaN (the call itself cannot see the device-side table and returns 0).
 * Scratch is a fixed array in the library image sized for K <= 32768 and 1..100 sites; larger
 * requests are rejected (status -7, message in fmc_last_error()).  The first call on a device
 * looks up that array's address and should come before any stream capture.  All calls share
 * the array, so calls that overlap on one GPU race.  Asynchronous on `stream` (a
 * cudaStream_t, NULL = default stream). */
int fmc_ewald1_guest_noalloc(int K, const int* kmax, const double* cell, const int* d_lmn, const double* d_akk,
                             const double* d_sk, int move, int nold, int nnew, const double* sites,
                             double recip_pref, double engsic, double* d_sk_new, double* d_engcpe, void* stream);

/* Host-only (no GPU needed): parse a deck and build its tables.  ints/dbls as in
 * fmc_chain_info (entries that need the device are zero).  Any of lmn[3K], akk[K], erc[mxgrid+1],
 * charges[framework atoms] may be NULL; *K and *nerc return the sizes. */
/* vdW table k (1-based, FIELD pair order; forgen, vdw_terms.f:190-396) of a deck: mxgrid+1
 * values; *ntables = tables including the zero table for undefined pairs. */
int fmc_deck_vdw(const char* dir, int k, double* out, int* ntables);
int fmc_deck_inspect(const char* dir, int* ints, double* dbls, int* lmn, double* akk, double* erc, double* charges,
                     int* K, int* nerc);
/* Host only: the same lists as fmc_batch_voxels, built on the host by testing every framework
 * atom against every voxel centre (voxel_edge <= 0: 2 A). */
int fmc_deck_voxels(const char* dir, double voxel_edge, int* nvox, int* off, int* atoms, long long cap,
                    long long* n_entries);

#ifdef __cplusplus
}
#endif

#endif /* FASTMC_B200_H */
