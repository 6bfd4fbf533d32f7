"""The streaming .npz writer (host only)."""

import numpy as np
import pytest

from idi_b200.simulation.output import NpzStream


@pytest.mark.parametrize("compress", [True, False])
def test_npz_stream_round_trip(tmp_path, compress):
    g = np.random.default_rng(0)
    data = g.normal(size=(7, 5, 3))
    path = tmp_path / "out.npz"
    with NpzStream(path, compress=compress) as npz:
        m = npz.array("result", data.shape, np.float64)
        for a, b in ((0, 3), (3, 4), (4, 7)):
            m.write(data[a:b])
        npz.add("settings", np.array([{"Ndet": 5}, ["fcc"]], dtype=object))
        npz.add("n", 7)
    f = np.load(path, allow_pickle=True)
    np.testing.assert_array_equal(f["result"], data)
    assert f["settings"][0]["Ndet"] == 5 and int(f["n"]) == 7


def test_npz_stream_checks_rows(tmp_path):
    npz = NpzStream(tmp_path / "bad.npz")
    m = npz.array("result", (3, 2), np.float32)
    m.write(np.zeros((2, 2)))
    with pytest.raises(ValueError):
        m.write(np.zeros((2, 2)))
    with pytest.raises(ValueError):
        m.write(np.zeros((1, 3)))
    with pytest.raises(ValueError):
        npz.close()
