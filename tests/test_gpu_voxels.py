"""Neighbour lists built on the device against the same lists built on the host.

The batched and serving kernels read a framework's candidate atoms from per-voxel lists (the
reference gathers them per trial in guestlistgen, utility_pack.f:3113-3177): every atom within
rcut + the voxel's circumradius of the voxel centre by true minimum image, ascending atom
index.  For orthorhombic cells the device skips the FP64 test of atoms whose voxel lies beyond
a conservative reach along some axis; the lists must still equal, entry for entry, the host's
test of every atom against every voxel."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

DECKS = ["small", "large", "ortho0", "ortho1", "ortho2", "calf20", "imcon4", "imcon5", "imcon6", "imcon7"]


def _same_lists(fmc, directory, edge):
    b = fmc.Batch([directory], [(1, 2, 3, 4)], voxel_edge=edge)
    nv_d, off_d, at_d = b.voxels(0)
    nv_h, off_h, at_h = fmc.deck_voxels(directory, edge)
    assert nv_d == nv_h
    assert np.array_equal(off_d, off_h)
    assert np.array_equal(at_d, at_h)
    return int(off_h[-1])


@pytest.mark.parametrize("edge", [2.0, 1.7, 1.0])
@pytest.mark.parametrize("name", DECKS)
def test_device_voxel_lists_equal_host(fmc, decks, name, edge):
    assert _same_lists(fmc, decks[name], edge) > 0


def test_voxel_lists_with_atoms_outside_the_cell(fmc, tmp_path):
    """Framework coordinates given anywhere (shifted by -L/2 and +1.3 L): the prefilter bins
    each atom by its wrapped position."""
    from fastmc_b200 import synth

    fw = synth.batched_frameworks(2, seed=5)[1]
    L = np.diag(fw.cell)
    xyz = fw.xyz.copy()
    xyz[::2] -= 0.5 * L
    xyz[1::3] += 1.3 * L
    moved = type(fw)(fw.cell, fw.names, xyz, fw.charges, fw.lj)
    d = synth.write_inputs(str(tmp_path / "moved"), moved, ["CO2"], [1.0], 298.0,
                           tuple(synth.kmax_for(x) for x in L))
    for edge in (2.0, 1.3):
        assert _same_lists(fmc, d, edge) > 0


def test_serving_request_voxel_lists(fmc, tmp_path):
    """Cubic request frameworks of the serving workload (400-6000 atoms)."""
    from fastmc_b200 import synth

    for r in synth.serving_requests(3, seed=11):
        d = synth.write_request(str(tmp_path / f"req{r['id']}"), r)
        assert _same_lists(fmc, d, 2.0) > 0
