/* A C caller of the drop-in ABI, written the way a host code in C (or a Fortran code through
 * bind(C)) calls it: the header alone, plain arrays, error codes and fmc_last_error.
 *
 *   dropin host  <deck>                 host-only entry points (no GPU)
 *   dropin chain <deck> <x y z ...>     one insertion pass and its commit on the GPU; prints the
 *                                       energies for the caller to compare
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "fastmc_b200.h"

static int fail(const char* what, int rc) {
  fprintf(stderr, "%s failed (%d): %s\n", what, rc, fmc_last_error());
  return 1;
}

int main(int argc, char** argv) {
  if (argc < 3) return 2;
  const char* deck = argv[2];
  if (strcmp(argv[1], "host") == 0) {
    int ints[16], K = 0, nerc = 0;
    double dbls[16];
    int rc = fmc_deck_inspect(deck, ints, dbls, NULL, NULL, NULL, NULL, &K, &nerc);
    if (rc) return fail("fmc_deck_inspect", rc);
    long long bytes = 0;
    double cost = 0.0;
    rc = fmc_deck_footprint(deck, 2.0, &bytes, &cost);
    if (rc) return fail("fmc_deck_footprint", rc);
    int nt = fmc_batch_tiles(NULL, NULL, NULL, 0);
    /* where node 0 would continue from if CONTROL said `restart` */
    char revive[1024], outdir[1024];
    int prev = -1;
    int restart_rc = fmc_restart_branch(deck, 0, revive, (int)sizeof(revive), outdir, (int)sizeof(outdir), &prev);
    if (restart_rc < 0) return fail("fmc_restart_branch", restart_rc);
    /* a directory that holds no deck: an error code and a message, no crash */
    rc = fmc_deck_inspect("/nonexistent-deck-directory", ints, dbls, NULL, NULL, NULL, NULL, &K, &nerc);
    printf("{\"K\": %d, \"nerc\": %d, \"imcon\": %d, \"bytes\": %lld, \"move_cost\": %.6f, \"tiles\": %d, "
           "\"restart_rc\": %d, \"prevnodes\": %d, \"revive\": \"%s\", \"outdir\": \"%s\", "
           "\"missing_rc\": %d, \"missing_msg\": %d}\n",
           K, nerc, ints[0], bytes, cost, nt, restart_rc, prev, revive, outdir, rc,
           (int)(strlen(fmc_last_error()) > 0));
    return 0;
  }
  if (strcmp(argv[1], "chain") == 0) {
    int natms = (argc - 3) / 3;
    if (natms < 1 || natms > 8) return 2;
    double xyz[24];
    for (int i = 0; i < 3 * natms; i++) xyz[i] = atof(argv[3 + i]);
    const int seed[4] = {12, 34, 56, 78};
    fmc_chain* c = NULL;
    int rc = fmc_chain_open(deck, seed, 0, &c);
    if (rc) return fail("fmc_chain_open", rc);
    double ewld1 = 0.0, ewld2 = 0.0, vdw = 0.0;
    rc = fmc_ewald1_guest(c, 0, natms, xyz, FMC_INSERT, 1, &ewld1);
    if (!rc) rc = fmc_guest_realspace(c, 0, natms, xyz, -1, &ewld2, &vdw);
    if (!rc) rc = fmc_commit(c, FMC_INSERT, 0, -1, xyz);
    double after2 = 0.0, afterv = 0.0;
    /* the same sites again, now against the committed molecule's own sites excluded (mol 0) */
    if (!rc) rc = fmc_guest_realspace(c, 0, natms, xyz, 0, &after2, &afterv);
    if (rc) {
      fmc_chain_close(c);
      return fail("drop-in pass", rc);
    }
    printf("{\"ewld1\": %.17g, \"ewld2\": %.17g, \"vdw\": %.17g, \"ewld2_excl\": %.17g, \"vdw_excl\": %.17g}\n",
           ewld1, ewld2, vdw, after2, afterv);
    fmc_chain_close(c);
    return 0;
  }
  return 2;
}
