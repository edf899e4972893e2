"""On-device observables (the output manager's .dat columns) against the
oracle's restatement, and the oracle against hand-computed values."""
import numpy as np
import pytest

import oracle_py as O
import sopb
from helpers import spec


def _three_bead_spec():
    # beads 0-1 bonded at r0 = 3.8 (stretched to 4.3), 0-2 a native contact
    # (r0 = 6, now 6), 1-2 only repulsive (within the pair cutoff)
    x = np.array([[0.0, 0.0, 0.0], [4.3, 0.0, 0.0], [0.0, 6.0, 0.0]], np.float32)
    p = sopb.default_params(timestep=0.08, pairs_threshold=50.0, pairlist_cutoff=20.0, pairs_cutoff=20.0)
    return sopb.JobSpec(x, np.array([[0, 1]]), [3.8], np.array([[0, 2]]), [6.0], [1.5], p, seed=9), x, p


def test_oracle_observables_known_values():
    sp, x, p = _three_bead_spec()
    o = O.OracleJob(sp)
    o.rebuild(True, True)
    obs = o.observables()
    d = 4.3 - 3.8
    fene = -0.5 * p.kspring_cov * p.R_limit ** 2 * np.log(1 - d * d / p.R_limit ** 2)
    assert obs[1] == pytest.approx(fene, rel=1e-5)
    assert obs[2] == pytest.approx(1.5 * (1.0 - 2.0), rel=1e-5)           # eh (1 - 2) at r = r0
    r12 = np.hypot(4.3, 6.0)
    assert obs[3] == pytest.approx(p.el * (p.a / r12) ** 6, rel=1e-5)      # the one non-bonded pair
    assert obs[4] == pytest.approx(obs[1] + obs[2] + obs[3])
    assert obs[5] == 1                                                     # the native contact is intact
    rg = np.sqrt((4.3 ** 2 + 6.0 ** 2 + r12 ** 2) / 9.0)
    assert obs[6] == pytest.approx(rg, rel=1e-6)
    assert obs[0] == 0.0 and obs[7] == 0.0


@pytest.mark.gpu
@pytest.mark.parametrize("n,mode,kw", [(150, "clamp", {}), (400, "free", {}), (300, "indent", {}),
                                       (3000, "clamp", dict(pairs_threshold=30.0, max_possiblePairs=2048)),
                                       (200, "free", dict(hi_on=1, hi_a=1.9, hi_epsilon_freq=10, hi_capricious=0))])
def test_observables_match_oracle(gpu_ctx, n, mode, kw):
    sp = spec(n, 51, mode, **kw)
    g, o = gpu_ctx.job(sp), O.OracleJob(sp)
    gpu_ctx.run([g], 25)
    assert o.advance(25) == 0
    # the same state on both sides: the GPU's coordinates and temperature
    # accumulator into the oracle (its lists were built at step 20 from
    # coordinates within 1e-5 A of these)
    o.write(sopb.COORDS, g.read(sopb.COORDS))
    o.write(sopb.TEMP, g.read(sopb.TEMP))
    go, oo = g.read(sopb.OBSERVABLES), o.observables()
    assert go[0] == pytest.approx(oo[0], rel=1e-5)                 # T
    for q in (1, 2, 3, 4):                                          # energies
        assert go[q] == pytest.approx(oo[q], rel=2e-4, abs=1e-3)
    assert abs(go[5] - oo[5]) <= 1                                  # intact native contacts
    assert go[6] == pytest.approx(oo[6], rel=1e-5)                  # Rg
    if kw.get("hi_on"):
        assert go[7] == pytest.approx(oo[7], rel=1e-4)
    g.destroy()
