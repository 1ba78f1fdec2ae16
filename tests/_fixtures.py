"""Loading of the golden fixtures (tests/golden/*.npz, made by make_golden.py)."""
from __future__ import annotations

from pathlib import Path

import numpy as np

GOLDEN = Path(__file__).resolve().parent / "golden"

NARROW = ["narrow_sphere_in", "narrow_sphere_out", "narrow_chain_in", "narrow_chain_out", "narrow_periodic_in"]
DWI = ["dwi_c1", "dwi_c1_cells", "dwi_overlap", "dwi_overlap_3axis"]
# walkers started on box faces, edges, corners and cell boundaries (the oracle's pin)
EDGE = ["dwi_faces"]


def load(name: str) -> dict:
    with np.load(GOLDEN / f"{name}.npz", allow_pickle=False) as z:
        return {k: z[k] for k in z.files}


def oracle_geometry(case: dict):
    from oracle import oracle as oz
    from oracle.cells_oracle import padded_as_lists
    nseg = tuple(int(v) for v in case["nseg"])
    ncell = nseg[0] * nseg[1] * nseg[2]
    st, ct, it = padded_as_lists(int(case["K"]), case["segments"], ncell)
    return oz.Geometry(case["spheres"].astype(np.float32), int(case["nstructures"]), tuple(case["L"]), nseg,
                       st, ct, it, case["D"], case["T2"], dL=tuple(case["dL"]))


def dirs_of(case: dict) -> np.ndarray:
    if bool(case.get("three_axis", False)):
        return np.eye(3, dtype=np.float32)
    return case["dirs"].astype(np.float32)
