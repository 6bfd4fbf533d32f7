"""Host side of the FFT autocorrelation: the FFT lengths (``fastlen``)
against the reference's ``idi.util.fastlen`` and the ABI of its kernels."""

import numpy as np

from idi_b200.reconstruction.cusimple import fastlen


def test_fastlen_properties():
    for x in (1, 2, 13, 26, 97, 1000, 2049, 4097):
        n = fastlen(x)
        assert n >= x
        m = n
        for f in (2, 3, 5, 7, 11):
            while m % f == 0:
                m //= f
        assert m == 1
        assert all(fastlen(y) == n for y in range(x, n + 1))  # nothing smaller in between


def test_fastlen_matches_reference(reference):
    assert all(reference.util.fastlen(x) == fastlen(x) for x in range(1, 3000))
