"""batchrates (src/batchrates.jl:22-60): host-side planning of drift-rate batches."""
from __future__ import annotations

import math
from dataclasses import dataclass
from fractions import Fraction

from .zdtutils import growNr


@dataclass(frozen=True)
class RateRange:
    """An equally spaced range of normalised drift rates (Julia's range(start, step, len)),
    held exactly as rationals like the reference's Rational ranges."""

    start: Fraction
    step: Fraction
    length: int

    def __len__(self):
        return self.length

    def __getitem__(self, i):
        if i < 0:
            i += self.length
        if not 0 <= i < self.length:
            raise IndexError(i)
        return self.start + i * self.step

    def __iter__(self):
        return (self.start + i * self.step for i in range(self.length))

    @property
    def first(self):
        return self.start

    @property
    def last(self):
        return self.start + (self.length - 1) * self.step


def _round_nearest_even(x):
    return int(round(x))


def _round_from_zero(x):
    return int(math.copysign(math.ceil(abs(x)), x)) if x != 0 else 0


def _round_to_zero(x):
    return int(math.trunc(x))


def batchrates(Nt, dhzps, r1, r2=None, Nrb=360):
    """Split the drift span [r1, r2] Hz/s (step |dhzps| Hz/s) into equal-length batches of
    normalised rates with step 1/(Nt-1) (batchrates.jl:22-60).  Returns a list of
    RateRange, each suitable for ZDTWorkspace."""
    if r2 is None:
        r2 = -r1
    if r2 < r1:
        r1, r2 = r2, r1
    nc1 = _round_nearest_even(r1 / dhzps)
    nc2 = _round_nearest_even(r2 / dhzps)
    Nrspan = abs(nc2 - nc1) + 1
    Nrb = min(Nrb, Nrspan)
    Nrb = growNr(Nt, Nrb)
    Nr = -(-Nrspan // Nrb) * Nrb
    Nrbonus = Nr - Nrspan
    sgn = (dhzps > 0) - (dhzps < 0)
    nc1 -= _round_from_zero(sgn * Nrbonus / 2)
    nc2 += _round_to_zero(sgn * Nrbonus / 2)
    a = Fraction(nc1, Nt - 1)
    b = Fraction(nc2, Nt - 1)
    step = (b - a) / (Nr - 1) if Nr > 1 else Fraction(1, Nt - 1)
    if Nr % Nrb != 0:
        raise AssertionError(f"number of rates ({Nr}) is not divisible by Nrb ({Nrb})")
    return [RateRange(a + i * step, step, Nrb) for i in range(0, Nr, Nrb)]
