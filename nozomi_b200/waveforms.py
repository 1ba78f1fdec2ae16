"""Diffusion gradient waveforms (the protocol input of the walk).

Same classes, sample grids and amplitude conventions as the reference's
simulation_toolkit/simulation_engine/waveforms.py:
  * wave amplitude 1 == 100 mT/m (the walk scales it by 267.5e-4 per ms,
    diffsim3d.py:252-255);
  * PGSE samples t = dt, 2dt, ... te with strict lobe inequalities
    (waveforms.py:164-186), which makes the two lobes of a symmetric PGSE differ
    by one sample on some grids (20/10/30 at dt = 0.01: 999 and 1000 samples);
  * b-values from the cumulative sum of gamma * wave (waveforms.py:147-153),
    gamma = 267.513 rad/ms/mT.
The reference's DiffGradWaveform.calculate_bvalue reads a missing attribute
(``self.gwave``, waveforms.py:138-145); here it evaluates the same formula on
``self.wave`` scaled by gmax.
"""
from __future__ import annotations

import numpy as np

GAMMA = 267.513  # rad/ms/mT (waveforms.py:4)
DT0 = 0.0001     # default time step, ms (waveforms.py:6)


class DiffGradWaveform:
    wave: np.ndarray
    dt: float

    def calculate_bvalue_from_wave(self) -> float:
        """b of the unit waveform in ms/um^2: sum(cumsum(gamma * wave / 1e4)^2) * dt^3."""
        g_um = self.wave / 10e3
        return float(np.sum(np.cumsum(GAMMA * g_um) ** 2) * self.dt ** 3)

    def calculate_bvalue(self, gmax=None) -> float:
        if gmax is None:
            gmax = getattr(self, "gmax", 1.0)
        g_um = self.wave / 10e3
        return float(np.sum(np.cumsum(gmax * GAMMA * g_um) ** 2) * self.dt ** 3)

    def set_bvalues(self, b):
        b0 = self.calculate_bvalue(1)
        self.b = b
        self.gmax = np.sqrt(np.asarray(b) / b0)

    def set_gmax(self, gmax):
        self.gmax = gmax
        self.b = self.calculate_bvalue(gmax)

    def amplitude_for_b(self, b) -> np.ndarray:
        """Wave amplitude (units of 100 mT/m) that gives b (ms/um^2)."""
        return np.sqrt(np.asarray(b, np.float64) / self.calculate_bvalue_from_wave())


class PGDiffWaveform(DiffGradWaveform):
    """Pulsed-gradient spin echo: +1 lobe, then -1 lobe, of width little_delta,
    Delta apart, centred on te/2."""

    def __init__(self, big_delta, little_delta, te, time_step=DT0):
        self.big_delta = big_delta
        self.little_delta = little_delta
        self.te = te
        self.dt = time_step
        self.generate_waveform()

    def generate_waveform(self):
        self.t = np.arange(self.dt, self.te + self.dt, self.dt)
        self.wave = np.zeros_like(self.t)
        c1 = self.te / 2 - self.big_delta / 2
        c2 = self.te / 2 + self.big_delta / 2
        h = self.little_delta / 2
        self.wave[(self.t > c1 - h) & (self.t < c1 + h)] = 1
        self.wave[(self.t > c2 - h) & (self.t < c2 + h)] = -1


def _quarter(phase_frac):
    return phase_frac * (np.pi / 2)


class CosineOGDiffWaveform(DiffGradWaveform):
    """Cosine oscillating gradient: a quarter-sine ramp at twice the frequency,
    num_oscillations cosine periods, a quarter-cosine ramp down; then the
    negated copy centred on 3te/4 (waveforms.py:188-247)."""

    def __init__(self, num_oscillations, frequency, gmax, te, time_step=DT0):
        self.num_oscillations = num_oscillations
        self.frequency = frequency
        self.gmax = gmax
        self.te = te
        self.dt = time_step
        self.generate_waveform()

    def generate_waveform(self):
        self.t = np.arange(self.dt, self.te + self.dt, self.dt)
        self.wave = np.zeros_like(self.t)
        period = 1.0 / self.frequency * 1000
        cos_dur = self.num_oscillations * period
        ramp = period / 8
        half = cos_dur + 2 * ramp
        for sign, start in ((1.0, self.te / 4 - half / 2), (-1.0, 3 * self.te / 4 - half / 2)):
            for i, t in enumerate(self.t):
                if start <= t < start + ramp:
                    self.wave[i] = sign * self.gmax * np.sin((t - start) / ramp * np.pi / 2)
                elif start + ramp <= t < start + ramp + cos_dur:
                    self.wave[i] = sign * self.gmax * np.cos(2 * np.pi * self.frequency * (t - (start + ramp)))
                elif start + ramp + cos_dur <= t < start + 2 * ramp + cos_dur:
                    self.wave[i] = sign * self.gmax * np.cos((t - (start + ramp + cos_dur)) / ramp * np.pi / 2)


class ApodizedCosineOGSEWaveform(DiffGradWaveform):
    """Apodised cosine OGSE (Does et al. 2003): quarter sine at 2f, N cosine
    cycles, quarter cosine at 2f; f = (0.25 + N) / T (waveforms.py:250-343)."""

    def __init__(self, N_cycles, T_duration, te=None, gmax=1.0, time_step=DT0):
        self.N_cycles = N_cycles
        self.T_duration = T_duration
        self.gmax = gmax
        self.dt = time_step
        self.t_eff = T_duration / (4 * N_cycles)
        self.te = 4 * T_duration if te is None else te
        self.generate_waveform()

    def _durations(self):
        f_cos = (0.25 + self.N_cycles) / self.T_duration
        f_apod = 2 * f_cos
        return f_cos, f_apod, 0.25 / f_apod, self.N_cycles / f_cos

    def generate_waveform(self):
        self.t = np.arange(0, self.te + self.dt, self.dt)
        self.wave = np.zeros_like(self.t)
        _, _, apod, cos_dur = self._durations()
        self._lobe(self.te / 4 - self.T_duration / 2, 1.0, apod, cos_dur)
        self._lobe(3 * self.te / 4 - self.T_duration / 2, -1.0, apod, cos_dur)

    def _lobe(self, t_start, polarity, apod, cos_dur):
        for i, t in enumerate(self.t):
            tr = t - t_start
            if 0 <= tr < apod:
                self.wave[i] = polarity * self.gmax * np.sin((tr / apod) * (np.pi / 2))
            elif apod <= tr < apod + cos_dur:
                prog = (tr - apod) / cos_dur
                self.wave[i] = polarity * self.gmax * np.cos(2 * np.pi * self.N_cycles * prog)
            elif apod + cos_dur <= tr < 2 * apod + cos_dur:
                self.wave[i] = polarity * self.gmax * np.cos(((tr - (apod + cos_dur)) / apod) * (np.pi / 2))

    def get_effective_diffusion_time(self):
        return self.t_eff

    def get_waveform_info(self):
        f_cos, f_apod, apod, cos_dur = self._durations()
        return {"N_cycles": self.N_cycles, "T_duration_ms": self.T_duration,
                "effective_diffusion_time_ms": self.t_eff, "total_echo_time_ms": self.te,
                "apodization_duration_ms": apod, "cosine_duration_ms": cos_dur,
                "cosine_frequency_Hz": f_cos * 1000, "apodization_frequency_Hz": f_apod * 1000,
                "frequency_ratio": f_apod / f_cos}


class ArbitraryWaveform(DiffGradWaveform):
    """Any sampled waveform (amplitude 1 == 100 mT/m) on a uniform grid."""

    def __init__(self, wave, time_step):
        self.wave = np.asarray(wave, np.float64)
        self.dt = time_step
        self.t = self.dt * np.arange(1, self.wave.size + 1)


def step_tables(gwave) -> tuple[np.ndarray, np.ndarray]:
    """Per-step walk arguments exactly as DwiSim3d.simulate_multi_directions
    forms them (diffsim3d.py:250-255): G_n = wave_n * dt * 267.5 / 1e4 and
    G_area_n = cumulative trapezoid(wave) * dt * 267.7 / 1e4, both rounded to
    float32 when passed to the kernel."""
    wave = np.asarray(gwave.wave, np.float64)
    dt = gwave.dt
    area = np.zeros_like(wave)
    if wave.size > 1:
        area[1:] = np.cumsum((wave[1:] + wave[:-1]) / 2.0)
    area = area * dt
    # element by element the same float64 operations, in the same order, as
    # the reference's scalar expressions, then one rounding to float32
    G = (((wave * dt) * 267.5) / 10000).astype(np.float32)
    Ga = ((area * 267.7) / 10000).astype(np.float32)
    return G, Ga
