"""Keys this library adds to the reference's config format: the Python
config layer reads them into sopb_params, leaves the reference's keys and
the updater period alone, and the near-list skin defaults to 0 (4 A)."""
import os
import sys

import sopb_config as CFG

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
import ref_cases  # noqa: E402


def params(extra=""):
    return CFG.job_config(CFG.Config(text=ref_cases.config_text("pull2") + extra)).params


def test_verlet_skin_key():
    base, wide, off = params(), params("\nverlet_skin 6.5\n"), params("\nverlet_skin -1\n")
    assert base.verlet_skin == 0.0
    assert wide.verlet_skin == 6.5 and off.verlet_skin == -1.0
    assert base.stride == wide.stride == off.stride
    for key in ("timestep", "pairs_freq", "pairlist_cutoff", "possiblepairs_freq", "max_pairs"):
        assert getattr(base, key) == getattr(wide, key)


def test_hi_refresh_joins_the_updater_period():
    text = "\nhi_on on\nhi_exact on\nhi_a 1.9\nhi_refresh 7\n"
    p, base = params(text), params()
    assert p.hi_refresh == 7
    assert p.stride == min(base.stride, 7)              # the refresh is one more updater period
