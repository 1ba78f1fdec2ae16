"""Simulation geometry: structures of spheres in a box.

Same classes, attributes and semantics as the reference's
simulation_toolkit/simulation_engine/geometry.py:
  * ``Structure3D(x, y, z, r, D, T2, rho)`` (geometry.py:8-35): one structure
    (an axon) as a list of spheres, stored as column vectors;
  * ``SimGeometry3D(Lx, Ly, Lz, D, T2, rho)`` (:37-72): the box
    [-L/2, L/2]^3 holding structures; ``spheres`` is the SoA [5, S] array
    (cx, cy, cz, r, structure id), the box is the last entry of
    ``structures`` and has id ``nstructures``; lower ids take precedence where
    structures overlap.
``gpu_seed`` keeps the reference's signature (:73) but seeds with
nozomi_b200's seeding kernel: one launch with a bounded number of rounds,
an error instead of an endless loop when a target has no volume.
"""
from __future__ import annotations

import numpy as np


class Structure3D:
    """A structure made of spheres (geometry.py:8-35)."""

    def __init__(self, x, y, z, r, D, T2, rho):
        x = np.asarray(x)
        self.nspheres = x.size
        self.x = np.reshape(x, [self.nspheres, 1])
        self.y = np.reshape(np.asarray(y), [self.nspheres, 1])
        self.z = np.reshape(np.asarray(z), [self.nspheres, 1])
        self.r = np.reshape(np.asarray(r), [self.nspheres, 1])
        self.D = D
        self.T2 = T2
        self.rho = rho
        self.tol = 1e-4

    def isinside(self, rnd):
        """Per column of rnd [3, N]: inside any sphere of this structure."""
        rnd = np.asarray(rnd)
        inside = ((rnd[0, :] - self.x) ** 2 + (rnd[1, :] - self.y) ** 2 + (rnd[2, :] - self.z) ** 2
                  - self.r ** 2 < 0)
        return inside.any(axis=0)


class SimGeometry3D:
    """The box and its structures (geometry.py:37-72)."""

    def __init__(self, Lx, Ly, Lz, D, T2, rho):
        self.Lx = Lx
        self.Ly = Ly
        self.Lz = Lz
        self.nsphere = 0
        self.spheres = np.zeros([5, self.nsphere])
        self.nstructures = 0
        self.structures = [self]  # the last item is always the box
        self.D = D
        self.T2 = T2
        self.rho = rho

    def add_structure(self, struct: Structure3D):
        self.structures[-1] = struct
        self.structures.append(self)
        new = np.zeros([5, struct.nspheres])
        new[0, :] = struct.x.T
        new[1, :] = struct.y.T
        new[2, :] = struct.z.T
        new[3, :] = struct.r.T
        new[4, :] = self.nstructures
        self.spheres = np.concatenate([self.spheres, new], axis=1)
        self.nstructures += 1
        self.nsphere += struct.nspheres

    def isinside(self, rnd):
        rnd = np.asarray(rnd)
        return ((rnd[0, :] > -self.Lx / 2) & (rnd[1, :] > -self.Ly / 2) & (rnd[2, :] > -self.Lz / 2) &
                (rnd[0, :] < self.Lx / 2) & (rnd[1, :] < self.Ly / 2) & (rnd[2, :] < self.Lz / 2))

    # -- device helpers ------------------------------------------------------
    def D_array(self):
        return np.array([s.D for s in self.structures], np.float32)

    def T2_array(self):
        return np.array([s.T2 for s in self.structures], np.float32)

    def device_substrate(self, nseg=None, cell: float = 2.0, near_margin=None):
        """This geometry on the device, with cell lists (nseg per axis, or a
        grid of about `cell` um)."""
        from . import engine
        from .substrates import cell_grid
        L = (self.Lx, self.Ly, self.Lz)
        if nseg is None:
            nseg = cell_grid(L, cell)
        return engine.DeviceSubstrate(self.spheres, self.nstructures, L, nseg, self.D_array(), self.T2_array(),
                                      near_margin=near_margin)

    def gpu_seed(self, gpu_seed_kernel=None, nspin=0, structIdxs=None, seed=None, max_rounds=100000):
        """Seed `nspin` positions uniformly in the target structures
        (structIdxs; default all structures and the box).  Returns [3, nspin]
        float32.  ``gpu_seed_kernel`` is accepted for call compatibility with
        the reference and ignored."""
        from . import engine
        if structIdxs is None:
            structIdxs = np.arange(self.nstructures + 1)
        if seed is None:
            seed = int(np.random.randint(np.iinfo(np.int32).max))
        sub = self.device_substrate()
        spins, _ = engine.seed(sub, [int(i) for i in np.atleast_1d(structIdxs)], int(nspin), key=seed,
                               max_rounds=max_rounds)
        return spins.cpu().numpy()
