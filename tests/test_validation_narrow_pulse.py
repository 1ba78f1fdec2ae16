"""The reference's narrow-pulse validation suite
(tests/validation/narrow_pulse/test_01..03 of the reference), run through
nozomi_b200's drop-in API with the same geometries, walker counts, time step,
diffusivity, step counts and assertions (plots dropped).  The periodic
geometry (516 spheres) runs 20,000 of the reference's 50,000 steps on a
3 x 3 x 3 cell grid instead of the reference's single cell.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

pytest.importorskip("torch")


def _api():
    from nozomi_b200.diffsim3d import DiffSim3d
    from nozomi_b200.geometry import SimGeometry3D, Structure3D
    return DiffSim3d, SimGeometry3D, Structure3D


def _chain():
    nsphere = 20
    sz = np.arange(-nsphere / 2 - 2, nsphere / 2 + 3) * 10.0 / nsphere
    sy = np.sin(2 * np.pi * np.arange(-2, nsphere + 3) / nsphere) * 0.25
    return np.full(sz.shape, 0), sy, sz, np.full(sz.shape, 1)


def _outside(sg3, spins):
    inside = False
    for struct in sg3.structures[:-1]:
        inside = np.logical_or(inside, struct.isinside(spins))
    return np.invert(inside)


def test_free_diffusion_empty_arena():
    DiffSim3d, SimGeometry3D, _ = _api()
    Lx = Ly = Lz = 10
    D, T2, rho = 3.0, 100, 1
    sg3 = SimGeometry3D(Lx, Ly, Lz, D, T2, rho)
    dt, nt, spins = 0.002, 50000, 100000
    sim = DiffSim3d(sg3, spins)
    sim.set_segments()
    for n in range(nt):
        sim.step(dt)
    x = sim.spins_d.get()
    for a, L in ((0, Lx), (1, Ly), (2, Lz)):
        assert (-L / 2 <= x[a]).all() and (x[a] <= L / 2).all()
    msd = np.sum(((sim.spins_d[0, :] - sim.spins0_d[0, :]) ** 2).get() / spins)
    assert np.isclose(np.abs(msd / 2 / dt / nt), D, rtol=1e-1)


def test_inside_single_sphere():
    DiffSim3d, SimGeometry3D, Structure3D = _api()
    D, T2, rho = 3.0, 100, 1
    sg3 = SimGeometry3D(10, 10, 10, D, T2, rho)
    sp = Structure3D(np.array([0]), np.array([0]), np.array([0]), np.array([1]), D, T2, rho)
    sg3.add_structure(sp)
    dt, nt, spins = 0.002, 50000, 100000
    sim = DiffSim3d(sg3, spins)
    sim.set_segments()
    sim.setup(structures=[0])
    assert sp.isinside(sim.spins).all()
    for n in range(nt):
        sim.step(dt)
    assert sp.isinside(sim.spins_d.get()).all()


def test_outside_single_sphere():
    DiffSim3d, SimGeometry3D, Structure3D = _api()
    D, T2, rho = 3.0, 100, 1
    sg3 = SimGeometry3D(10, 10, 10, D, T2, rho)
    sg3.add_structure(Structure3D(np.array([0]), np.array([0]), np.array([0]), np.array([1]), D, T2, rho))
    dt, nt, spins = 0.002, 50000, 100000
    sim = DiffSim3d(sg3, spins)
    sim.set_segments()
    sim.setup(structures=[1])
    assert _outside(sg3, sim.spins_d.get()).all()
    for n in range(nt):
        sim.step(dt)
    assert _outside(sg3, sim.spins_d.get()).all()
    assert abs(np.mean(sim.sig_d.get()) - np.exp(-nt * dt / T2)) < 1e-2


def _msd_over_2t(sim, spins, dt, nt):
    return [np.sum(((sim.spins_d[a, :] - sim.spins0_d[a, :]) ** 2).get()) / spins / 2 / dt / nt for a in range(3)]


def test_inside_multiple_spheres():
    DiffSim3d, SimGeometry3D, Structure3D = _api()
    D, T2, rho = 3.0, 100, 1
    sg3 = SimGeometry3D(10.0, 10.0, 10.0, D, T2, rho)
    sg3.add_structure(Structure3D(*_chain(), D, T2, rho))
    dt, nt, spins = 0.002, 50000, 100000
    sim = DiffSim3d(sg3, spins)
    sim.set_segments()
    sim.setup(structures=[0])
    assert not _outside(sg3, sim.spins_d.get()).any()
    for n in range(nt):
        sim.step(dt)
    assert not _outside(sg3, sim.spins_d.get()).any()
    dx, dy, dz = _msd_over_2t(sim, spins, dt, nt)
    assert D - 0.2 < dz < D + 0.2
    assert dy < 0.2 and dx < 0.2
    assert abs(np.mean(sim.sig_d.get()) - np.exp(-nt * dt / T2)) < 1e-2


def test_outside_multiple_spheres():
    DiffSim3d, SimGeometry3D, Structure3D = _api()
    D, T2, rho = 3.0, 100, 1
    sg3 = SimGeometry3D(10, 10, 10, D, T2, rho)
    sg3.add_structure(Structure3D(*_chain(), D, T2, rho))
    dt, nt, spins = 0.002, 50000, 100000
    sim = DiffSim3d(sg3, spins)
    sim.set_segments()
    sim.setup(structures=[1])
    assert _outside(sg3, sim.spins_d.get()).all()
    for n in range(nt):
        sim.step(dt)
    assert _outside(sg3, sim.spins_d.get()).all()
    dx, dy, dz = _msd_over_2t(sim, spins, dt, nt)
    assert D - 0.2 < dz < D + 0.2
    assert dy > D - 0.5 and dx > D - 0.5
    assert abs(np.mean(sim.sig_d.get()) - np.exp(-nt * dt / T2)) < 1e-2


def _periodic_chains():
    Lz = 10.0
    z = np.linspace(-Lz / 2, Lz / 2, num=200)
    z = np.concatenate((z[-30:-1] - Lz, z, z[1:30] + Lz))
    y = np.concatenate((np.sin(2 * np.pi * z / 10.0),) * 2)
    x = np.concatenate((np.full(z.shape, 0) + 5.0, np.full(z.shape, 0) - 5.0))
    zz = np.concatenate((z, z))
    return x, y, zz, np.full(zz.shape, 1)


@pytest.mark.parametrize("inside", [True, False])
def test_periodic_boundary_xyz(inside):
    DiffSim3d, SimGeometry3D, Structure3D = _api()
    D, T2, rho = 3.0, 100, 1
    sg3 = SimGeometry3D(10.0, 10.0, 10.0, D, T2, rho)
    sg3.add_structure(Structure3D(*_periodic_chains(), D, T2, rho))
    dt, nt, spins = 0.002, 20000, 100000
    sim = DiffSim3d(sg3, spins)
    sim.set_segments(3, 3, 3)
    sim.setup(structures=[0] if inside else [1])
    for n in range(nt):
        sim.step(dt)
    out = _outside(sg3, sim.spins_d.get())
    dx, dy, dz = _msd_over_2t(sim, spins, dt, nt)
    if inside:
        assert not out.any()
        assert D - 0.5 < dz < D + 0.5
        assert dy < 0.2 and dx < 0.2
    else:
        assert out.all()
        assert D - 0.2 < dz < D + 0.2
        assert dy > D - 0.5 and dx > D - 0.5
    assert abs(np.mean(sim.sig_d.get()) - np.exp(-nt * dt / T2)) < 1e-2
