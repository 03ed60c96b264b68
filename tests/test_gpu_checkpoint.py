"""Checkpoint / resume through the engine: a run split at a .bfm checkpoint (positions plus the
draw-stream position in its header) equals the run straight through and the oracle."""
import numpy as np
import pytest

import pscbfm_b200 as P
from oracle import oracle as O
from pscbfm_b200 import systems as S

pytestmark = pytest.mark.gpu

MODES = {"graph": P.MODE_GRAPH, "resident": P.MODE_RESIDENT, "launch": P.MODE_LAUNCH, "persistent": P.MODE_PERSISTENT,
         "cluster": P.MODE_CLUSTER}


@pytest.mark.parametrize("mode", list(MODES))
@pytest.mark.parametrize("build", [S.small_chains, S.rings_and_free, S.crosslinked_network])
def test_resume_from_checkpoint(build, mode, tmp_path):
    s = build()
    if mode == "resident" and max(s.box) > 64:
        pytest.skip("box larger than the resident kernel holds")
    want, _ = O.run(s, 50)
    u = P.UpdaterGPUScBFM_AB_Type(0).load_system(s, mode=MODES[mode])
    u.runSimulationOnGPU(30)
    p = str(tmp_path / "ck.bfm")
    u.save_checkpoint(p, s)
    u.runSimulationOnGPU(20)
    assert np.array_equal(u.get_coords(), want)
    u.close()
    v, _ = P.UpdaterGPUScBFM_AB_Type.load_checkpoint(p, system=s, mode=MODES[mode])
    assert v.substep() == 30 * v.n_colors()[0]
    v.runSimulationOnGPU(20)
    assert np.array_equal(v.get_coords(), want)
    v.validate()
    v.close()


def test_set_substep_with_pending_marks():
    """Moving the stream position after a grid-phase run first clears that run's marks."""
    s = S.crosslinked_network()
    want, _ = O.run(s, 40, substep0=0)
    u = P.UpdaterGPUScBFM_AB_Type(0).load_system(s, mode=P.MODE_GRAPH)
    u.runSimulationOnGPU(25)
    t = u.substep()
    u.set_substep(t)
    u.runSimulationOnGPU(15)
    assert np.array_equal(u.get_coords(), want)
    u.validate()
    u.close()
