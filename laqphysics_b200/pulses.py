"""sin^2-envelope laser pulses in atomic units (host side; scalars per time step).

Drop-in for the reference's ``Pulse`` (python/pulses.py:5-48): the same fields
(omega, cycles, field = peak electric field F0, start, cep) with the same defaults, and
the same quantities E(t), A(t) = -int E dt, int envelope dt and int envelope^2 dt.

Derivation used here.  With s = t - start, T = 2 pi cycles / omega and b = 2 pi / T,

    E(s) = F0 sin^2(pi s / T) cos(omega s + cep)
         = F0 Re[ e^{i cep} (1/2 e^{i omega s} - 1/4 e^{i (omega + b) s} - 1/4 e^{i (omega - b) s}) ]

so A is a sum of three phasor integrals, each written as
int_0^u e^{i w s} ds = u e^{i w u / 2} sinc(w u / 2 pi), which stays exact when
omega - b -> 0 (one-cycle pulses).  The envelope integrals use the cosine series
sin^2 x = 1/2 - cos 2x / 2 and sin^4 x = 3/8 - cos 2x / 2 + cos 4x / 8.  For an integer
number (>= 2) of cycles the analytic final A is zero for any CEP; the value is set to
exactly zero after the pulse so that no rounding residue acts as an impulse.
"""
import math
from dataclasses import dataclass

import numpy as np

# E(s) / F0 = Re[e^{i cep} sum_k weight_k exp(i (omega + shift_k b) s)]
_PHASORS = ((.5, 0), (-.25, 1), (-.25, -1))
# sin^2(pi s/T) and sin^4(pi s/T) as sum_k a_k cos(k b s)
_SIN2 = (.5, -.5)
_SIN4 = (.375, -.5, .125)


@dataclass(frozen=True)
class Pulse:
    omega: float = 1.5
    cycles: float = 60
    field: float = .0534
    start: float = 0.
    cep: float = 0.

    def __post_init__(self):
        values = (self.omega, self.cycles, self.field, self.start, self.cep)
        if not all(np.isfinite(v) for v in values):
            raise ValueError(f'pulse parameters must be finite, got {values}')
        if self.omega <= 0 or self.cycles <= 1 or self.field < 0 or self.start < 0:
            raise ValueError('a pulse needs omega > 0, more than one cycle, field >= 0 and start >= 0')

    @property
    def duration(self):
        return 2 * np.pi * self.cycles / self.omega

    def _elapsed(self, t):
        """Time since the start, clipped to the pulse window."""
        return np.clip(np.asarray(t) - self.start, 0, self.duration)

    def envelope(self, t):
        s = np.asarray(t) - self.start
        inside = (s >= 0) & (s <= self.duration)
        return np.where(inside, np.sin(np.pi * s / self.duration) ** 2, 0.)

    def electric(self, t):
        phase = self.omega * (np.asarray(t) - self.start) + self.cep
        return self.field * self.envelope(t) * np.cos(phase)

    def vector(self, t):
        """A(t) = -int_start^t E(t') dt' in closed form (phasor integrals above)."""
        if isinstance(t, (float, int)):
            return self._vector_scalar(float(t))
        u = self._elapsed(t)
        b = 2 * np.pi / self.duration
        total = 0.
        for weight, shift in _PHASORS:
            w = self.omega + shift * b
            # Re[e^{i cep} int_0^u e^{i w s} ds]
            total = total + weight * u * np.sinc(w * u / (2 * np.pi)) * np.cos(self.cep + w * u / 2)
        A = -self.field * total
        whole = round(self.cycles)
        if whole >= 2 and abs(self.cycles - whole) < 1e-12:
            A = np.where(np.asarray(t) >= self.start + self.duration, 0., A)
        return A

    def _vector_scalar(self, t):
        """vector() for one time with the math module (a time-step loop calls it every step):
        sinc(w u / 2 pi) = sin(x) / x with x = w u / 2."""
        u = min(max(t - self.start, 0.), self.duration)
        b = 2 * math.pi / self.duration
        total = 0.
        for weight, shift in _PHASORS:
            x = (self.omega + shift * b) * u / 2
            total += weight * u * (math.sin(x) / x if x != 0 else 1.) * math.cos(self.cep + x)
        whole = round(self.cycles)
        if whole >= 2 and abs(self.cycles - whole) < 1e-12 and t >= self.start + self.duration:
            return 0.
        return -self.field * total

    def _cosine_series_integral(self, t, coefficients):
        """int_0^u sum_k a_k cos(k b s) ds with u = elapsed time, b = 2 pi / T."""
        u = self._elapsed(t)
        b = 2 * np.pi / self.duration
        total = coefficients[0] * u
        for k, a in enumerate(coefficients[1:], start=1):
            total = total + a * np.sin(k * b * u) / (k * b)
        return total

    def area_envelope(self, t):
        """int_start^t envelope dt'."""
        return self._cosine_series_integral(t, _SIN2)

    def area_squared(self, t):
        """int_start^t envelope^2 dt'."""
        return self._cosine_series_integral(t, _SIN4)
