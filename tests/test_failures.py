"""Failure handling that needs no GPU: the host-side substrate checks that run
before any device work (a bad substrate is refused with a NozomiError naming
the problem instead of walking garbage)."""
import numpy as np
import pytest


def _ok():
    sph = np.array([[0.0, 1.0], [0.0, 0.0], [0.0, 0.0], [0.5, 0.7], [0.0, 1.0]])
    return sph, 2, (4.0, 4.0, 4.0), (2, 2, 2), [2.0, 2.0, 2.0], [100.0, 100.0, 100.0]


@pytest.mark.parametrize("mutate, msg", [
    (lambda a: a[0].__setitem__((3, 1), np.nan), "non-finite centre or radius"),
    (lambda a: a[0].__setitem__((0, 0), np.inf), "non-finite centre or radius"),
    (lambda a: a[0].__setitem__((3, 0), 0.0), "radius <= 0"),
    (lambda a: a[0].__setitem__((3, 1), -1.0), "radius <= 0"),
    (lambda a: a[0].__setitem__((4, 1), 2.0), "structure id"),
    (lambda a: a[0].__setitem__((4, 1), 0.5), "structure id"),
    (lambda a: a.__setitem__(2, (4.0, 0.0, 4.0)), "box"),
    (lambda a: a.__setitem__(3, (2, 0, 2)), "cell grid"),
    (lambda a: a.__setitem__(4, [2.0, 2.0]), "one entry per structure"),
    (lambda a: a.__setitem__(4, [2.0, -1.0, 2.0]), "D must be"),
    (lambda a: a.__setitem__(5, [100.0, 0.0, 100.0]), "T2 must be"),
])
def test_bad_substrates_are_refused(mutate, msg):
    from nozomi_b200.engine import NozomiError, validate_substrate
    args = list(_ok())
    validate_substrate(*args)
    args[0] = args[0].copy()
    mutate(args)
    with pytest.raises(NozomiError, match=msg):
        validate_substrate(*args)


def test_empty_substrate_is_valid():
    from nozomi_b200.engine import validate_substrate
    validate_substrate(np.zeros((5, 0)), 0, (4.0, 4.0, 4.0), (1, 1, 1), [2.0], [100.0])
