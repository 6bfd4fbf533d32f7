"""simulate_to_npz: intensities streamed from the device pipeline into an
.npz equal |E|^2 of simulate on the same emitters."""

import numpy as np
import pytest

from idi_b200.simulation import cuda as sim
from idi_b200.simulation.simobj import fixed
from tests.helpers import rng, sphere

pytestmark = pytest.mark.gpu


def test_simulate_to_npz_matches_simulate(tmp_path):
    g = rng(41)
    n, nimg, ndet = 64, 9, 1024  # 72 MB of intensities: the pipeline runs in chunks
    pos = sphere(g, n, 0.01)
    ph = g.uniform(0, 2 * np.pi, (nimg, n))
    mk = lambda: fixed(6400.0, pos, ph)  # noqa: E731
    E = sim.simulate(nimg, mk(), ndet, 75.0, 1e5, settings="nf double", verbose=False)
    path = tmp_path / "run.npz"
    done = sim.simulate_to_npz(path, nimg, mk(), ndet, 75.0, 1e5, settings="nf double", verbose=False,
                               extra={"settings": np.array(["nf double"])})
    assert done == nimg
    f = np.load(path)
    assert f["result"].shape == (nimg, ndet, ndet) and str(f["settings"][0]) == "nf double"
    np.testing.assert_allclose(f["result"], np.square(np.abs(E)), rtol=1e-14, atol=0)
