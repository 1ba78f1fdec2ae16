"""The oracle against the reference's own outputs (golden fixtures).

The fixtures were produced by the reference's Python engine and kernel source
(tests/golden/make_golden.py); the C oracle must reproduce every float bit for
bit: positions, spins0, T2 signal, phase; the numpy cell-list restatement must
reproduce DiffSim3d.set_segments exactly; the seeding rule must accept exactly
the positions seedSpinsKernel accepts.
"""
import numpy as np
import pytest

from tests._fixtures import DWI, EDGE, NARROW, dirs_of, load, oracle_geometry
from oracle import oracle as oz
from oracle.cells_oracle import cells_members, segments_reference


@pytest.mark.parametrize("name", NARROW)
def test_narrow_pulse_bit_exact(name):
    c = load(name)
    g = oracle_geometry(c)
    spins = c["x0"].copy()
    spins0 = spins.copy()
    sig = np.ones(int(c["N"]), np.float32)
    r = oz.walk_f32(g, oz.philox(int(c["key"])), oz.MODE_SIG, spins, spins0, 0, int(c["nt"]), float(c["dt"]),
                    sig=sig)
    np.testing.assert_array_equal(spins, c["spins"])
    np.testing.assert_array_equal(spins0, c["spins0"])
    # T2 weighting goes through expf (glibc here, the reference's libm there): ulps only
    np.testing.assert_allclose(sig, c["sig"], rtol=2e-6)
    assert (r["flags"] & oz.FLAG_DRAWS_EXHAUSTED).sum() == 0


@pytest.mark.parametrize("name", DWI + EDGE)
def test_dwi_phase_bit_exact(name):
    c = load(name)
    g = oracle_geometry(c)
    N = int(c["N"])
    dirs = dirs_of(c)
    spins = c["x0"].astype(np.float32).copy()
    spins0 = spins.copy()
    phase = np.zeros((dirs.shape[1], N), np.float32)
    oz.walk_f32(g, oz.philox(int(c["key"])), oz.MODE_PHASE, spins, spins0, 0, int(c["nt"]), float(c["dt"]),
                G=c["G"], Garea=c["Garea"], phase=phase, diffdir=dirs)
    np.testing.assert_array_equal(spins, c["spins"])
    np.testing.assert_array_equal(spins0, c["spins0"])
    np.testing.assert_array_equal(phase, c["phase"])


def test_three_axis_equals_identity_directions():
    """randomWalk3d_phase (fixed x, y, z) is randomWalk3d_phase_multidirr with
    the identity as directions."""
    c = load("dwi_overlap_3axis")
    assert c["phase"].shape[0] == 3


def test_segments_match_set_segments():
    z = np.load(__import__("tests._fixtures", fromlist=["GOLDEN"]).GOLDEN / "segments.npz")
    for i in range(int(z["ncase"])):
        K, seg = segments_reference(z[f"case{i}_spheres"], tuple(z[f"case{i}_L"]), tuple(z[f"case{i}_nseg"]))
        assert K == int(z[f"case{i}_K"])
        np.testing.assert_array_equal(seg, z[f"case{i}_segments"])
    for name in NARROW + DWI + EDGE:
        c = load(name)
        nseg = tuple(int(v) for v in c["nseg"])
        K, seg = segments_reference(c["spheres"], tuple(c["L"]), nseg)
        assert K == int(c["K"])
        _assert_same_up_to_ties(c["spheres"], tuple(c["L"]), nseg, K, seg, c["segments"])


def _assert_same_up_to_ties(spheres, L, nseg, K, mine, ref):
    """The reference's unstable argsort may pick a different pad among spheres
    with equal in_segment; members must agree and pads must tie."""
    from oracle.cells_oracle import in_segment
    nx, ny, nz = nseg
    mine, ref = mine.reshape(-1, K), ref.reshape(-1, K)
    for n in range(nx):
        for m in range(ny):
            for p in range(nz):
                c = p * nx * ny + m * nx + n
                v = in_segment(spheres, L, nseg, (n, m, p))
                members = set(np.nonzero(v < 1.0)[0])
                assert members <= set(mine[c]) and members <= set(ref[c])
                np.testing.assert_array_equal(np.sort(v[mine[c]]), np.sort(v[ref[c]]))


def test_members_are_subset_of_padded_lists():
    z = np.load(__import__("tests._fixtures", fromlist=["GOLDEN"]).GOLDEN / "segments.npz")
    for i in range(int(z["ncase"])):
        nseg = tuple(int(v) for v in z[f"case{i}_nseg"])
        st, ct, it = cells_members(z[f"case{i}_spheres"], tuple(z[f"case{i}_L"]), nseg)
        K = int(z[f"case{i}_K"])
        assert ct.max() == K
        seg = z[f"case{i}_segments"].reshape(-1, K)
        for c in range(seg.shape[0]):
            assert set(it[st[c]:st[c] + ct[c]]) <= set(seg[c])


def test_seeding_rule_matches_seedSpinsKernel():
    from tests._fixtures import GOLDEN
    z = np.load(GOLDEN / "seeding.npz")
    L = tuple(z["L"])
    sph = z["spheres"]
    st, ct, it = cells_members(sph, L, (1, 1, 1))
    g = oz.Geometry(sph.astype(np.float32), 3, L, (1, 1, 1), st, ct, it, np.full(4, 2.0, np.float32),
                    np.full(4, 100.0, np.float32))
    u = z["u"]
    pos = ((u.T - np.float32(0.5)) * np.array(L, np.float32)[:, None]).astype(np.float32)
    for t in ("intra", "extra", "s1", "all"):
        acc = oz.seed_accept(g, z[f"{t}_targets"], pos)
        np.testing.assert_array_equal(acc, z[f"{t}_accept"])
        np.testing.assert_array_equal(pos[:, acc], z[f"{t}_pos"][:, acc])


def _packed_reference():
    """The reference kernel's CPU build for the packed substrate, its oracle
    geometry over the same padded table, and the seeded start positions."""
    import sys
    from pathlib import Path
    from oracle.build import reference_named
    from oracle.cells_oracle import padded_as_lists
    sys.path.insert(0, str(Path(__file__).resolve().parents[1]))
    import bench
    if reference_named("packed_cpu_16k") is None:
        pytest.skip("oracle/_ref reference build absent (the reference tree was absent at build)")
    sub, pg, dirs, _ = bench.workload_packed()
    ref = bench.ReferenceCpu("packed_cpu_16k", sub, pg, dirs)
    _, pars = reference_named("packed_cpu_16k")
    nseg = (int(pars["nLx"]), int(pars["nLy"]), int(pars["nLz"]))
    st, ct, it = padded_as_lists(ref.K, ref.seg, nseg[0] * nseg[1] * nseg[2])
    ns = sub.nstructures
    g = oz.Geometry(sub.spheres().astype(np.float32), ns, sub.L, nseg, st, ct, it,
                    np.full(ns + 1, 2.0, np.float32), np.full(ns + 1, 100.0, np.float32),
                    dL=(float(pars["dLx"]), float(pars["dLy"]), float(pars["dLz"])))
    return ref, g, pg, dirs, ref.spins.reshape(3, ref.N).copy()


def test_oracle_equals_reference_kernel_on_packed_substrate():
    """The headline substrate (200 packed beaded axons, 29,628 spheres with
    images, 40x40x80 um, 1 um cells, the reference's padded table K = 45):
    the reference's own randomWalk3d_phase_multidirr (sim3d_kernel.cu:719-943,
    compiled for the CPU with the template DiffSim3d fills in) and the oracle
    walk 16,000 seeded walkers through the first 400 waveform samples (the
    first gradient lobe, 30 directions) with the same Philox draws: positions,
    spins0 and phase bit for bit."""
    ref, g, pg, dirs, x0 = _packed_reference()
    N, nsteps = ref.N, 400
    ref.run(nsteps)
    spins, spins0 = x0.copy(), x0.copy()
    phase = np.zeros((dirs.shape[1], N), np.float32)
    oz.walk_f32(g, oz.philox(1000), oz.MODE_PHASE, spins, spins0, 0, nsteps, float(pg.dt), G=ref.G, Garea=ref.Ga,
                phase=phase, diffdir=dirs.astype(np.float32))
    np.testing.assert_array_equal(spins, ref.spins.reshape(3, N))
    np.testing.assert_array_equal(spins0, ref.spins0.reshape(3, N))
    np.testing.assert_array_equal(phase, ref.phase.reshape(-1, N))
    # and not trivially: the walkers moved and accrued phase
    assert np.abs(spins - x0).max() > 0.5 and np.abs(phase).max() > 0


@pytest.mark.parametrize("kernel", ["randomWalk3d", "randomWalk3d_phase"])
def test_oracle_equals_reference_narrow_and_three_axis_kernels_on_packed_substrate(kernel):
    """The reference's other two walks on the same substrate and build, 300
    steps of 16,000 walkers with the same Philox draws: randomWalk3d
    (sim3d_kernel.cu:340-522, T2 weighting) against the oracle's SIG mode
    (positions bit for bit, sig to expf ulps), and randomWalk3d_phase
    (:524-717, fixed x, y, z) against the oracle's PHASE mode with the
    identity as directions (bit for bit)."""
    import ctypes
    ref, g, pg, _, x0 = _packed_reference()
    N, nsteps, dt = ref.N, 300, float(pg.dt)
    P, f, i = ctypes.c_void_p, ctypes.c_float, ctypes.c_int
    lib = ref.lib
    spins = x0.reshape(-1).copy()  # the reference walks these in place; x0 stays the start
    spins0 = spins.copy()
    if kernel == "randomWalk3d":
        lib.ref_run_walk.argtypes = [i, i, i, f, P, P, P, P, P]
        sig_ref = np.ones(N, np.float32)
        for n in range(nsteps):
            lib.ref_run_walk(N // 1000, 1000, n, dt, ref.sph.ctypes.data, ref.seg.ctypes.data, spins.ctypes.data,
                             spins0.ctypes.data, sig_ref.ctypes.data)
        x, x00, sig = x0.copy(), x0.copy(), np.ones(N, np.float32)
        oz.walk_f32(g, oz.philox(1000), oz.MODE_SIG, x, x00, 0, nsteps, dt, sig=sig)
        np.testing.assert_allclose(sig, sig_ref, rtol=2e-6)
        assert sig.min() < 1.0
    else:
        lib.ref_run_walk_phase.argtypes = [i, i, i, f, P, P, P, P, P, f, f]
        ph_ref = np.zeros(3 * N, np.float32)
        for n in range(nsteps):
            lib.ref_run_walk_phase(N // 1000, 1000, n, dt, ref.sph.ctypes.data, ref.seg.ctypes.data,
                                   spins.ctypes.data, spins0.ctypes.data, ph_ref.ctypes.data, f(ref.G[n]),
                                   f(ref.Ga[n]))
        x, x00, ph = x0.copy(), x0.copy(), np.zeros((3, N), np.float32)
        oz.walk_f32(g, oz.philox(1000), oz.MODE_PHASE, x, x00, 0, nsteps, dt, G=ref.G, Garea=ref.Ga, phase=ph,
                    diffdir=np.eye(3, dtype=np.float32))
        np.testing.assert_array_equal(ph, ph_ref.reshape(3, N))
        assert np.abs(ph).max() > 0
    np.testing.assert_array_equal(x, spins.reshape(3, N))
    np.testing.assert_array_equal(x00, spins0.reshape(3, N))
    assert np.abs(x - x0).max() > 0.5
