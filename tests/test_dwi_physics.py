"""DWI signals against analytic oracles, through the drop-in API.

* free diffusion: S(b) = exp(-b D), b from the waveform's own discrete sum
  (waveforms.calculate_bvalue_from_wave);
* spins inside a sphere: Gaussian-phase approximation for PGSE (Murday &
  Cotts 1968, J. Chem. Phys. 48:4938), exact in the low-q limit used here;
* the fused DWI path against the per-step path: identical trajectories,
  phases equal to within FP32 rounding of the per-step sums.

Tolerances: 3 Monte Carlo standard errors of the signal plus the stated model
error (0.2 % for free diffusion's discrete b, 1 % for the sphere's GPA at
S > 0.6).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _dwi(L, structs, N, D, seed, dirs=None):
    from nozomi_b200.diffsim3d import DwiSim3d
    from nozomi_b200.geometry import SimGeometry3D, Structure3D
    sg3 = SimGeometry3D(*L, D, 1e9, 1)
    for s in structs:
        sg3.add_structure(Structure3D(*s, D, 1e9, 1))
    sim = DwiSim3d(sg3, N, diffdir=dirs)
    return sim, sg3


def _mc_sigma(S, N):
    # per-walker cos has variance (1 + S(2b) - 2 S(b)^2) / 2 <= 1/2
    return np.sqrt(0.5 / N)


def test_free_diffusion_signal():
    from nozomi_b200.waveforms import PGDiffWaveform
    D, N = 2.0, 200_000
    pg = PGDiffWaveform(20.0, 10.0, 30.0, time_step=0.005)
    b1 = pg.calculate_bvalue_from_wave()
    bvals = np.array([0.0, 0.25, 0.5, 1.0])
    amps = np.sqrt(bvals / b1)
    dirs = np.eye(3)
    sim, _ = _dwi((200.0, 200.0, 200.0), [], N, D, 3, dirs=dirs)
    sim.set_segments(4, 4, 4)
    sim.setup(initstates_int=11)
    S = sim.signal(pg, amplitudes=amps)
    ref = np.exp(-bvals * D)
    err = np.abs(S.real - ref[None, :])
    tol = 3 * _mc_sigma(ref, N) + 2e-3 * ref
    assert np.all(err <= tol[None, :]), (S.real, ref)
    assert np.all(np.abs(S.imag) < 3 * _mc_sigma(ref, N) + 1e-3)


def _murday_cotts(q, R, D, delta, Delta, nroots=60):
    """ln S = -2 q^2 sum_m [2 delta / (a D) - (2 + e^{-a D (Delta - delta)}
    - 2 e^{-a D delta} - 2 e^{-a D Delta} + e^{-a D (Delta + delta)}) / (a D)^2]
    / (a (a R^2 - 2)),  a = (mu_m / R)^2, mu_m the roots of j1'(mu) = 0;
    q in rad / (ms um) (gamma G)."""
    from scipy.optimize import brentq
    from scipy.special import spherical_jn
    f = lambda x: spherical_jn(1, x, derivative=True)  # noqa: E731
    roots, x = [], 0.5
    while len(roots) < nroots:
        if f(x) * f(x + 0.05) < 0:
            roots.append(brentq(f, x, x + 0.05))
        x += 0.05
    s = 0.0
    for mu in roots:
        a = (mu / R) ** 2
        aD = a * D
        num = 2 + np.exp(-aD * (Delta - delta)) - 2 * np.exp(-aD * delta) - 2 * np.exp(-aD * Delta) \
            + np.exp(-aD * (Delta + delta))
        s += (2 * delta / aD - num / aD ** 2) / (a * (a * R ** 2 - 2))
    return np.exp(-2 * q ** 2 * s)


def test_restricted_sphere_gpa():
    from nozomi_b200.waveforms import PGDiffWaveform
    D, N, R = 2.0, 200_000, 3.0
    pg = PGDiffWaveform(20.0, 10.0, 30.0, time_step=0.005)
    amps = np.array([0.0, 0.5, 1.0, 1.5])
    sim, _ = _dwi((10.0, 10.0, 10.0), [(np.array([0.0]), np.array([0.0]), np.array([0.0]), np.array([R]))],
                  N, D, 5, dirs=np.eye(3))
    sim.set_segments()
    sim.setup(structures=[0], initstates_int=21)
    S = sim.signal(pg, amplitudes=amps).real.mean(axis=0)  # isotropic: average x, y, z
    # the walk's unit: G per sample = 267.5e-4 * wave * dt -> q = 267.5e-4 rad/(ms um) per unit amplitude
    q = amps * 267.5e-4
    lob = (pg.wave == 1)
    delta = lob.sum() * pg.dt
    ref = np.array([_murday_cotts(qq, R - 1e-4, D, delta, 20.0) for qq in q])
    sig = 3 * np.sqrt(0.5 / (3 * N))
    assert np.all(ref[1:] > 0.6)
    np.testing.assert_allclose(S, ref, atol=sig + 0.01)


def test_fused_dwi_equals_per_step_dwi():
    from nozomi_b200.waveforms import PGDiffWaveform
    from nozomi_b200.substrates import beaded_axon
    sub = beaded_axon()
    pg = PGDiffWaveform(2.0, 1.0, 3.0, time_step=0.01)
    dirs = np.array([[1.0, 0.0, 0.6], [0.0, 0.0, 0.0], [0.0, 1.0, 0.8]])
    out = []
    for exact in (True, False):
        from nozomi_b200.diffsim3d import DwiSim3d
        g = sub.geometry(D=2.0)
        sim = DwiSim3d(g, 3000, diffdir=dirs)
        sim.set_segments(1, 1, 4)
        sim.setup(structures=[0], initstates_int=5)
        ph = sim.simulate_multi_directions(pg, exact=exact)
        out.append((ph, sim.spins_d.get(), sim.spins0_d.get()))
    (pe, xe, x0e), (pf, xf, x0f) = out
    np.testing.assert_array_equal(xe, xf)
    np.testing.assert_array_equal(x0e, x0f)
    scale = np.abs(pe).max() + 1e-6
    assert np.abs(pe - pf).max() <= 1e-5 * scale
