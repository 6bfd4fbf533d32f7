"""The oracle (CPU restatement) against the reference: committed golden
fixtures always, and the live reference code where its tree is present."""

import numpy as np
import pytest

import oracle
from tests.helpers import atoms, rel_field_err, rng, sphere, E_EV, K64


def _geom_from_meta(meta, settings):
    nx, ny, ps, dz, a0, a1, o0, o1, k = meta
    return oracle.geometry([int(nx), int(ny)], ps, dz, k, (a0, a1), (o0, o1)), oracle.flags_from_settings(settings)


def test_oracle_forward_matches_golden(golden_forward):
    names = sorted({k.split("__")[0] for k in golden_forward.files})
    assert len(names) >= 6
    for name in names:
        g, f = _geom_from_meta(golden_forward[f"{name}__meta"], str(golden_forward[f"{name}__settings"]))
        pos = golden_forward[f"{name}__pos"]
        ph = golden_forward[f"{name}__phases"]
        ref = golden_forward[f"{name}__field"]
        for i in range(ph.shape[0]):
            E = oracle.wavefield(g, f, atoms(pos, ph[i]))
            if name in ("ff", "nf", "nf_rot_off"):
                # same rounding sequence as the numba kernel: bit-exact but for rare 1-ulp pixels
                assert np.mean(E == ref[i]) > 0.99, name
            assert rel_field_err(E, ref[i]) < 1e-12, name


def test_oracle_time_matches_golden(golden_time):
    names = sorted({k.split("__")[0] for k in golden_time.files})
    for name in names:
        nx, ny, ps, dz, a0, a1, c, tau, pw, k = golden_time[f"{name}__meta"]
        settings = str(golden_time[f"{name}__settings"])
        g = oracle.geometry([int(nx), int(ny)], ps, dz, k, (a0, a1))
        f = oracle.flags_from_settings(settings)
        at = atoms(golden_time[f"{name}__pos"], golden_time[f"{name}__phases"][0])
        times = golden_time[f"{name}__times"]
        img = oracle.time_image(g, f, at, times, c, tau)
        ref = golden_time[f"{name}__image"]
        assert np.max(np.abs(img - ref) / np.abs(ref)) < 1e-12, name
        keys = golden_time[f"{name}__keys"]
        sk = golden_time[f"{name}__sorted_keys"]
        for p in range(int(nx) * int(ny)):
            t, _ = oracle.time_keys(g, f, at, times, c, p // int(ny), p % int(ny))
            assert np.array_equal(t, keys[p]), (name, p)  # arrival keys bit-exact
            order = oracle.time_order(g, f, at, times, c, p // int(ny), p % int(ny))
            assert np.array_equal(t[order], sk[p]), (name, p)  # same sorted sequence


def test_oracle_matches_live_reference(reference):
    g0 = rng(77)
    n = 250
    pos = sphere(g0, n, 0.012)
    ph = g0.uniform(0, 2 * np.pi, (1, n))
    from oracle import refshim

    for settings in ["nf", "", "nf scale"]:
        obj = refshim.InjectedObject(E_EV, pos, ph)
        ref = reference.cpu.simulate(1, obj, [10, 14], 70.0, 9e4, K64, settings=settings)[0]
        E = oracle.wavefield(oracle.geometry([10, 14], 70.0, 9e4, K64), oracle.flags_from_settings(settings),
                             atoms(pos, ph[0]))
        assert rel_field_err(E, ref) < 1e-12
        if settings == "nf":
            assert np.array_equal(E, ref)


def test_oracle_rotation_matches_reference(reference):
    for a in [(0.1, 0.2, 0.0), (1.3, -0.7, 0.0), (0.5, 0.01, 0.3)]:
        assert np.array_equal(oracle.rotation(*a), reference.util.rotation(*a))


@pytest.mark.parametrize("settings", ["nf", "", "secondorder", "nf scale", "scale"])
def test_oracle_adjoint_finite_differences(settings):
    """The adjoint restatement (no reference code) against central differences."""
    g0 = rng(5)
    n = 12
    pos = sphere(g0, n, 0.01)
    ph = g0.uniform(0, 2 * np.pi, n)
    amp = g0.uniform(0.5, 1.5, n)
    geo = oracle.geometry([6, 5], 3000.0, 1e5, K64, (0.05, 0.02), (100.0, -50.0))
    f = oracle.flags_from_settings(settings)
    target = np.abs(oracle.wavefield(geo, f, atoms(pos + 2e-5 * g0.normal(size=pos.shape), ph), amp)) ** 2

    def loss(p, q, a):
        E = oracle.wavefield(geo, f, atoms(p, q), a)
        return np.sum((np.abs(E) ** 2 - target) ** 2)

    E = oracle.wavefield(geo, f, atoms(pos, ph), amp)
    L, gpos, gpsi, gamp = oracle.adjoint(geo, f, atoms(pos, ph), amp, E, target)
    assert np.isclose(L, loss(pos, ph, amp))
    # the near-field phase follows the reference's |d - r| - d_z form, whose
    # FP64 rounding (k * ulp(|d|) ~ 5e-7 rad) is noise for small steps
    h = 1e-6 if "nf" in settings else 1e-7
    tol = 2e-3 if "nf" in settings else 1e-5
    for j in range(0, n, 3):
        for d in range(3):
            p1 = pos.copy(); p1[j, d] += h
            p2 = pos.copy(); p2[j, d] -= h
            fd = (loss(p1, ph, amp) - loss(p2, ph, amp)) / (2 * h)
            assert abs(fd - gpos[j, d]) <= tol * np.abs(gpos).max(), (j, d)
        q1 = ph.copy(); q1[j] += 1e-6
        q2 = ph.copy(); q2[j] -= 1e-6
        fd = (loss(pos, q1, amp) - loss(pos, q2, amp)) / 2e-6
        assert abs(fd - gpsi[j]) <= tol * np.abs(gpsi).max()
        a1 = amp.copy(); a1[j] += 1e-6
        a2 = amp.copy(); a2[j] -= 1e-6
        fd = (loss(pos, ph, a1) - loss(pos, ph, a2)) / 2e-6
        assert abs(fd - gamp[j]) <= tol * np.abs(gamp).max()


def test_intensity_metrics_planted_error():
    """The error metric catches a planted error on the oracle side."""
    g0 = rng(3)
    I_ref = g0.exponential(1.0, 10000)
    I = I_ref.copy()
    I[17] *= 1 + 3e-4
    m = oracle.intensity_metrics(I, I_ref)
    assert m["max_rel_masked"] > 2e-4 or I_ref[17] < 1e-3
    assert oracle.intensity_metrics(I_ref, I_ref)["max_rel_masked"] == 0.0
