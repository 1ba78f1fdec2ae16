"""Physics of the walk rule against an analytic result, on the CPU.

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
