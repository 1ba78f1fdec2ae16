"""Waveforms and per-step protocol tables against the reference's own
(waveforms.py samples and b-values; the G / G_area arguments recorded from
DwiSim3d.simulate_multi_directions in the golden runs)."""
import numpy as np

from tests._fixtures import GOLDEN, load
from nozomi_b200 import waveforms as wf


def test_waveform_samples_match_reference():
    z = np.load(GOLDEN / "waveforms.npz")
    pg = wf.PGDiffWaveform(20.0, 10.0, 30.0, time_step=0.01)
    np.testing.assert_array_equal(pg.wave, z["pgse_20_10_30_dt01"])
    assert pg.calculate_bvalue_from_wave() == z["pgse_20_10_30_dt01_b1"]
    assert (pg.wave == 1).sum() == 999 and (pg.wave == -1).sum() == 1000
    pg5 = wf.PGDiffWaveform(20.0, 10.0, 30.0, time_step=0.005)
    np.testing.assert_array_equal(pg5.wave, z["pgse_20_10_30_dt005"])
    assert pg5.calculate_bvalue_from_wave() == z["pgse_20_10_30_dt005_b1"]
    np.testing.assert_array_equal(wf.PGDiffWaveform(40.0, 10.0, 78.0, time_step=0.002).wave, z["pgse_40_10_78_dt002"])
    og = wf.CosineOGDiffWaveform(2, 50.0, 1.0, 60.0, time_step=0.01)
    np.testing.assert_array_equal(og.wave, z["cos_ogse_2_50_60_dt01"])
    assert og.calculate_bvalue_from_wave() == z["cos_ogse_2_50_60_dt01_b1"]
    ap = wf.ApodizedCosineOGSEWaveform(2, 20.0, te=50.0, time_step=0.01)
    np.testing.assert_array_equal(ap.wave, z["apod_ogse_2_20_50_dt01"])
    assert ap.calculate_bvalue_from_wave() == z["apod_ogse_2_20_50_dt01_b1"]


def test_step_tables_match_reference_driver():
    for name in ("dwi_c1", "dwi_overlap"):
        c = load(name)
        gw = wf.ArbitraryWaveform(c["wave"], float(c["dt"]))
        gw.dt = 0.01  # the reference passes the waveform's python float dt
        G, Ga = wf.step_tables(gw)
        np.testing.assert_array_equal(G, c["G"])
        np.testing.assert_array_equal(Ga, c["Garea"])


def test_bvalue_fix_and_amplitudes():
    pg = wf.PGDiffWaveform(20.0, 10.0, 30.0, time_step=0.005)
    b1 = pg.calculate_bvalue_from_wave()
    assert abs(pg.calculate_bvalue(1.0) - b1) < 1e-12
    assert abs(pg.calculate_bvalue(2.0) - 4 * b1) < 1e-9
    a = pg.amplitude_for_b([0, 1, 2, 3])
    np.testing.assert_allclose(a ** 2 * b1, [0, 1, 2, 3])
