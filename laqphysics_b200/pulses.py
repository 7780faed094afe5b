"""sin^2 laser pulses; E = -dA/dt, F0 = peak electric field (a.u.).

Same conventions as the reference's ``Pulse`` (python/pulses.py:5-48): the vector
potential is the exact time integral of the specified electric field, written with
sinc so that it stays accurate when omega approaches the envelope frequency, and a
pulse with an integer number (>=2) of cycles has exactly zero final A.
"""
from dataclasses import dataclass

import numpy as np


@dataclass(frozen=True)
class Pulse:
    omega: float = 1.5
    cycles: float = 60
    field: float = .0534
    start: float = 0.
    cep: float = 0.

    def __post_init__(self):
        finite = np.all(np.isfinite([self.omega, self.cycles, self.field, self.start, self.cep]))
        if not finite or self.omega <= 0 or self.cycles <= 1 or self.field < 0 or self.start < 0:
            raise ValueError('finite omega>0, cycles>1, field>=0, start>=0 and finite CEP are required')

    @property
    def duration(self):
        return 2 * np.pi * self.cycles / self.omega

    def envelope(self, t):
        s = np.asarray(t) - self.start
        return np.where((s >= 0) & (s <= self.duration), np.sin(np.pi * s / self.duration) ** 2, 0.)

    def electric(self, t):
        return self.field * self.envelope(t) * np.cos(self.omega * (np.asarray(t) - self.start) + self.cep)

    def vector(self, t):
        """A(t) = -int_start^t E; sin^2 = 1/2 - cos(b s)/2 splits E into three cosines."""
        u = np.clip(np.asarray(t) - self.start, 0, self.duration)
        b = 2 * np.pi / self.duration

        def cos_integral(w):
            # int_0^u cos(cep + w s) ds = u cos(cep + w u/2) sinc(w u / 2pi)
            return u * np.cos(self.cep + w * u / 2) * np.sinc(w * u / (2 * np.pi))

        value = -self.field * (.5 * cos_integral(self.omega) - .25 * cos_integral(self.omega + b)
                               - .25 * cos_integral(self.omega - b))
        if round(self.cycles) >= 2 and abs(self.cycles - round(self.cycles)) < 1e-12:
            value = np.where(np.asarray(t) >= self.start + self.duration, 0., value)
        return value

    def area_envelope(self, t):
        u = np.clip(np.asarray(t) - self.start, 0, self.duration)
        return u / 2 - self.duration * np.sin(2 * np.pi * u / self.duration) / (4 * np.pi)

    def area_squared(self, t):
        u = np.clip(np.asarray(t) - self.start, 0, self.duration)
        T = self.duration
        return 3 * u / 8 - T * np.sin(2 * np.pi * u / T) / (4 * np.pi) + T * np.sin(4 * np.pi * u / T) / (32 * np.pi)
