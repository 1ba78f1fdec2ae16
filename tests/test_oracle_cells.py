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
