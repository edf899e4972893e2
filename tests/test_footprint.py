"""sopb_job_footprint (host arithmetic, no GPU needed): the device bytes a
job takes, which the serving loop admits by, include the buffers of the
path the job runs on -- the exact-HI tensor, the HI per-bead buffers and the
grid near list for grid-path jobs, the bitmask lists for resident jobs."""
import sopb
from helpers import spec


def a256(v):
    return (v + 255) // 256 * 256


def fp(n, mode="clamp", **kw):
    return spec(n, 3, mode, **kw).footprint()


def test_exact_hi_counts_its_tensor():
    n = 1500
    ld = (3 * n + 31) // 32 * 32            # leading dimension above 128 beads
    tiles = (3 * n + 127) // 128
    # two 128 x 128 inverse buffers, and the TF32 hi and lo planes of two
    # outer panels of 4 tile columns (the default policy)
    chol = 2 * 128 * 128 * 4 + 2 * (2 * tiles * 128 * 4 * 128 * 4)
    grow = fp(n, hi_on=1, hi_exact=1, hi_a=1.9, hi_capricious=0) - fp(n, grid_path=1)
    assert grow >= 3 * n * ld * 4 + chol
    assert grow < 3 * n * ld * 4 + chol + 64 * n * 16     # plus the per-bead HI buffers and slices


def test_tea_counts_its_per_bead_buffers():
    n = 4000
    grow = fp(n, hi_on=1, hi_a=1.9, hi_capricious=0) - fp(n, grid_path=1)
    assert grow >= 4 * n * 16 + n * 4


def test_grid_near_list_is_counted_once():
    n = 3000                                 # max_pairs 512, max_possiblePairs 4096 -> 1024 near entries
    cap_nr = 1024
    with_near = fp(n, grid_path=1)
    without = fp(n, grid_path=1, verlet_skin=-1.0)
    assert with_near - without == a256(n * cap_nr * 4) + a256(n * 4) + a256(n * 16)


def test_resident_job_counts_masks_not_rows():
    n = 300
    W = (n + 31) // 32
    resident, grid = fp(n), fp(n, grid_path=1)
    assert resident < grid
    # the resident layout holds two n x W masks where the grid path holds
    # n x cap_pp possible-pair rows (cap_pp = n - 1 here)
    assert resident >= 2 * n * W * 4
    assert grid - resident >= n * (n - 1) * 4 - 2 * a256(n * W * 4) - a256(n * (n - 1) * 2)
