"""The C cell-list builder of the oracle against the numpy restatement."""
import numpy as np

from tests._fixtures import GOLDEN
from oracle import oracle as oz
from oracle.cells_oracle import cells_members


def test_c_cells_match_numpy():
    z = np.load(GOLDEN / "segments.npz")
    for i in range(int(z["ncase"])):
        sph, L3, nseg = z[f"case{i}_spheres"], tuple(z[f"case{i}_L"]), tuple(int(v) for v in z[f"case{i}_nseg"])
        a = cells_members(sph, L3, nseg)
        b = oz.cells(sph, L3, nseg)
        for x, y in zip(a, b):
            np.testing.assert_array_equal(x, y)


def test_c_padded_table_matches_numpy():
    """oz_segments (the C padded table used at full size) against the numpy
    restatement of set_segments on the golden cases and a 12-axon bundle."""
    from oracle.cells_oracle import segments_reference
    from nozomi_b200.substrates import axon_bundle, cell_grid
    z = np.load(GOLDEN / "segments.npz")
    cases = [(z[f"case{i}_spheres"], tuple(z[f"case{i}_L"]), tuple(int(v) for v in z[f"case{i}_nseg"]))
             for i in range(int(z["ncase"]))]
    sub = axon_bundle(12, seed=5)
    cases.append((sub.spheres(), sub.L, cell_grid(sub.L, 1.0)))
    for sph, L3, nseg in cases:
        K, seg = segments_reference(sph, L3, nseg)
        np.testing.assert_array_equal(oz.segments(sph, L3, nseg, K), seg)


def test_window_member_counts_match_c_cells():
    """The baseline build's windowed member count (K of the reference
    kernel's template) against the oracle's cell lists."""
    from baseline.reference_gpu import member_counts
    from nozomi_b200.substrates import axon_bundle, beaded_axon, cell_grid
    for sub, nseg in ((beaded_axon(), (1, 1, 8)), (axon_bundle(25, seed=1), None)):
        nseg = nseg or cell_grid(sub.L, 0.5)
        np.testing.assert_array_equal(member_counts(sub.spheres(), sub.L, nseg), oz.cells(sub.spheres(), sub.L, nseg)[1])
