"""FFT length selection (blond/toolbox/next_regular.py:9-59).

The rule is reproduced exactly because it fixes ``n_fft`` and therefore the
circular-convolution length of the induced voltage: a target <= 6 or a power
of two is returned as is; otherwise the result is twice the smallest
5-smooth (2^a 3^b 5^c) number that is >= ceil(target / 2).
"""
from __future__ import annotations


def _smallest_5smooth_at_least(t: int) -> int:
    best = None
    p5 = 1
    while True:
        p35 = p5
        while True:
            # smallest power of two q with p35 * q >= t
            q = 1
            while p35 * q < t:
                q *= 2
            cand = p35 * q
            if best is None or cand < best:
                best = cand
            if p35 >= t:
                break
            p35 *= 3
        if p5 >= t:
            break
        p5 *= 5
    return best


def next_regular(target: int) -> int:
    target = int(target)
    if target <= 6:
        return target
    if target & (target - 1) == 0:
        return target
    return 2 * _smallest_5smooth_at_least(-(-target // 2))
