"""int64 observables on the device equal the numpy int64 recomputation from the positions
(per-molecule sums for Rg^2, end-to-end Ree^2, bond-vector histogram, displacement sum)."""
import numpy as np
import pytest

import pscbfm_b200 as P
from oracle import oracle as O
from pscbfm_b200 import systems as S

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("build", [S.small_chains, S.rings_and_free, S.crosslinked_network,
                                   lambda: S.serpentine_chains(64, 128, 0.4, seed=13)])
def test_observables_exact(build):
    s = build()
    u = P.UpdaterGPUScBFM_AB_Type(0)
    u.load_system(s)
    assert np.array_equal(u.observables_raw(), O.observables(s, s.xyz, s.xyz))
    u.runSimulationOnGPU(150)
    xyz = u.get_coords().copy()
    ref, _ = O.run(s, 150)
    assert np.array_equal(xyz, ref)
    raw = u.observables_raw()
    assert np.array_equal(raw, O.observables(s, xyz, s.xyz))
    obs = P.updater.decode_observables(raw, u.molecule_sizes())
    assert obs["msd"] > 0 and np.isfinite(obs["rg2_mean"])
    assert int(obs["bond_hist"].sum()) == int(s.nbr_count.sum())
    u.reset_msd_reference()
    assert u.observables()["msd_sum"] == 0
    u.close()


def test_molecule_numbering():
    s = S.rings_and_free()
    u = P.UpdaterGPUScBFM_AB_Type(0)
    u.load_system(s)
    sizes = u.molecule_sizes()
    mol = O.molecules(s)
    assert np.array_equal(sizes, np.bincount(mol))
    u.close()
