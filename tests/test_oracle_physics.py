"""Physics of the walk rule against analytic results, on the CPU.

The oracle is bit-exact with the reference's kernel and with the product's
walks, so these hold for both.  Three checks: free diffusion's exp(-bD) and
the restricted sphere's Gaussian-phase signal (the GPU versions of both run
through the drop-in API in tests/test_dwi_physics.py), and the reference's
own calibration target below.

The reference calibrates its walker count and time step against the radial
diffusivity inside a cylinder (tests/calibration/num_molecules_and_time_step_
calibration/calibration_for_num_molecules_and_time_step_search.py:35-89 and
:105-131): Burcaw et al. 2015 (after Stepisnik 1993 and Callaghan 1995),

    D_perp(t) = a^2 / (4t) - (2 a^2 / t) sum_k exp(-b_k^2 D0 t / a^2) / (b_k^2 (b_k^2 - 1)),

b_k the roots of J1'.  Here the oracle (bit-exact with the reference's
kernel and with the product's walks) walks 12,000 walkers seeded inside a
cylinder built as the reference builds one: spheres of the cylinder's radius
every 0.2 um along z, z-periodic with images.  Per-axis D(t) = sum dx^2 /
(2 t N), the reference's moment definition (sim3d_kernel.cu:162-238), is
checked at six times from 0.2 to 10 ms: radial within 5 % of Burcaw's D(t)
(the estimate's standard error is about 1 %), axial within 5 % of D0."""
import numpy as np
from scipy.special import jnp_zeros

from oracle import oracle as oz
from oracle.cells_oracle import cells_members


def burcaw_dperp(t, a, D0, terms=100):
    b = jnp_zeros(1, terms)
    s = np.sum(np.exp(-b ** 2 * D0 * t / a ** 2) / (b ** 2 * (b ** 2 - 1)))
    return a ** 2 / (4 * t) - (2 * a ** 2 / t) * s


def test_cylinder_radial_diffusivity_matches_burcaw():
    a, D0, Lz, spacing = 2.0, 2.0, 20.0, 0.2
    L = (8.0, 8.0, Lz)
    z = -Lz / 2 + spacing / 2 + spacing * np.arange(int(round(Lz / spacing)))
    z = np.concatenate([z - Lz, z, z + Lz])
    z = z[np.abs(z) < Lz / 2 + a + 1.5]  # z-periodic images reaching into the box
    sph = np.zeros((5, z.size))
    sph[2], sph[3] = z, a
    nseg = (1, 1, 20)
    st, ct, it = cells_members(sph, L, nseg)
    g = oz.Geometry(sph.astype(np.float32), 1, L, nseg, st, ct, it, np.full(2, D0, np.float32),
                    np.full(2, 100.0, np.float32))
    N, dt = 12_000, 0.002
    x, _, left = oz.seed(g, [0], N, 7)
    assert left == 0
    spins, spins0 = x.copy(), x.copy()
    done = 0
    for T in (0.2, 0.5, 1.0, 2.0, 5.0, 10.0):
        n = int(round(T / dt))
        oz.walk_f32(g, oz.philox(11), oz.MODE_SIG, spins, spins0, done, n - done, dt, sig=np.ones(N, np.float32),
                    counters=False)
        done = n
        m = oz.moments(spins, spins0)
        D = m[:3] / (2 * T * N)
        want = burcaw_dperp(T, a, D0)
        assert abs(0.5 * (D[0] + D[1]) / want - 1) < 0.05, (T, D, want)
        assert abs(D[2] / D0 - 1) < 0.05, (T, D)
    # every walker stayed inside the cylinder (containment is exact)
    assert np.hypot(spins[0], spins[1]).max() < a


def _phase_walk(sph, nstructures, L, nseg, targets, N, D, pg, key):
    """Oracle phase walk along x, y, z of N seeded walkers: phase [3, N]."""
    from nozomi_b200.waveforms import step_tables
    st, ct, it = cells_members(sph, L, nseg)
    g = oz.Geometry(np.asarray(sph, np.float32).reshape(5, -1), nstructures, L, nseg, st, ct, it,
                    np.full(nstructures + 1, D, np.float32), np.full(nstructures + 1, 1e9, np.float32))
    x, _, left = oz.seed(g, targets, N, key ^ 0x5EED)
    assert left == 0
    G, Ga = step_tables(pg)
    spins, spins0 = x.copy(), x.copy()
    phase = np.zeros((3, N), np.float32)
    oz.walk_f32(g, oz.philox(key), oz.MODE_PHASE, spins, spins0, 0, G.size, pg.dt, G=G, Garea=Ga, phase=phase,
                diffdir=np.eye(3, dtype=np.float32), counters=False)
    return phase


def test_free_diffusion_signal_oracle():
    """S(b) = exp(-b D) on an empty arena, b from the waveform's own discrete
    sum, PGSE 20/10/30 ms at dt = 10 us: within 3 Monte Carlo standard errors
    plus 0.2 % (the discrete b)."""
    from nozomi_b200.waveforms import PGDiffWaveform
    D, N = 2.0, 20_000
    pg = PGDiffWaveform(20.0, 10.0, 30.0, time_step=0.01)
    b1 = pg.calculate_bvalue_from_wave()
    bvals = np.array([0.0, 0.25, 0.5, 1.0])
    phase = _phase_walk(np.zeros((5, 0)), 0, (200.0, 200.0, 200.0), (1, 1, 1), [0], N, D, pg, 3)
    S = oz.signal_phase(phase, np.sqrt(bvals / b1))
    ref = np.exp(-bvals * D)
    tol = 3 * np.sqrt(0.5 / N) + 2e-3 * ref
    assert np.all(np.abs(S.real - ref[None, :]) <= tol[None, :]), (S.real, ref)
    assert np.all(np.abs(S.imag) <= 3 * np.sqrt(0.5 / N) + 1e-3)


def test_restricted_sphere_gpa_oracle():
    """Walkers inside a sphere of radius 3 um, PGSE 20/10/30 ms: the Gaussian
    phase approximation (Murday & Cotts 1968) at S > 0.6, averaged over x, y
    and z, within 3 standard errors plus 1 % (the approximation)."""
    from nozomi_b200.waveforms import PGDiffWaveform
    from tests.test_dwi_physics import _murday_cotts
    D, N, R = 2.0, 20_000, 3.0
    pg = PGDiffWaveform(20.0, 10.0, 30.0, time_step=0.01)
    amps = np.array([0.0, 0.5, 1.0, 1.5])
    sph = np.array([[0.0], [0.0], [0.0], [R], [0.0]])
    phase = _phase_walk(sph, 1, (10.0, 10.0, 10.0), (1, 1, 1), [0], N, D, pg, 21)
    S = oz.signal_phase(phase, amps).real.mean(axis=0)
    q = amps * 267.5e-4
    delta = (pg.wave == 1).sum() * pg.dt
    ref = np.array([_murday_cotts(qq, R - 1e-4, D, delta, 20.0) for qq in q])
    assert np.all(ref[1:] > 0.6)
    np.testing.assert_allclose(S, ref, atol=3 * np.sqrt(0.5 / (3 * N)) + 0.01)
