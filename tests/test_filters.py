"""Row filters beyond Ram-Lak (CPU): the oracle's filter spectra and the
product's exact Toeplitz taps (b2t_filter_taps) against the reference's own
genFilter output (tests/golden/filters_reference.npz, made by
make_filter_golden.py from the reference build), and the custom
projection / sinogram / rprojection / rsinogram types against the oracle."""
import importlib
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "filters_reference.npz")


def _golden():
    g = np.load(GOLDEN)
    for key in g.files:
        name, N, d, p = key.split('|')
        yield name, int(N), float(d), float(p), g[key].astype(np.float64)


def test_oracle_spectra_match_reference(orc):
    worst = 0.0
    for name, N, d, p, G in _golden():
        ours = orc.filter_spectrum(name, N, d, p)
        err = np.abs(ours - G).max() / np.abs(G).max()
        worst = max(worst, err)
        assert err < 1e-5, (name, N, d, p, err)
    assert worst > 0.0  # the fixtures are float: a bit-equal match would be suspicious


@pytest.mark.parametrize("N", [128, 256, 2048])
def test_product_taps_match_reference(astra, orc, N):
    P = importlib.import_module("astra-toolbox_b200.projector")
    n = N // 2 - 3  # nextpow2(2 n) == N
    for name, gN, d, p, G in _golden():
        if gN != N:
            continue
        want = orc._spectrum_taps(G, N, n)
        got = P.filter_taps(P.FilterSpec(name, d=d, parameter=p), n)[0]
        err = np.abs(got - want).max() / np.abs(want).max()
        assert err < 1e-5, (name, N, d, p, err)


def test_ramlak_taps_are_the_closed_form(astra, orc):
    P = importlib.import_module("astra-toolbox_b200.projector")
    for n in (5, 64, 301, 832):
        t = orc.ramp_taps(n)
        want = np.concatenate([t[:0:-1], t])
        got = P.filter_taps('ram-lak', n)[0]
        assert np.abs(got - want).max() < 1e-6 * 0.5


def test_custom_filter_taps(astra, orc):
    P = importlib.import_module("astra-toolbox_b200.projector")
    rng = np.random.default_rng(7)
    n, views = 37, 5
    F = 128 // 2 + 1  # nextpow2(2 * 37) = 128 -> 65 bins
    spec1 = rng.random(F).astype(np.float32)
    specs = rng.random((views, F)).astype(np.float32)
    sp1 = rng.standard_normal(9).astype(np.float32)
    sps = rng.standard_normal((views, 12)).astype(np.float32)
    cases = [('projection', spec1, 1), ('sinogram', specs, views), ('rprojection', sp1, 1),
             ('rsinogram', sps, views)]
    for name, custom, sets in cases:
        got = P.filter_taps(P.FilterSpec(name, custom=custom), n, views)
        want = orc.filter_taps(name, n, views, custom=custom)
        assert got.shape == (sets, 2 * n - 1), name
        assert np.abs(got - want).max() <= 1e-6 * max(1.0, np.abs(want).max()), name
    # the spatial filter lands centred: element W // 2 at offset 0
    got = P.filter_taps(P.FilterSpec('rprojection', custom=sp1), n)[0]
    assert got[n - 1] == sp1[len(sp1) // 2] and got[n - 1 + 3] == sp1[len(sp1) // 2 + 3]
    # wrong custom sizes are refused, as the reference's checkCustomFilterSize does
    with pytest.raises(astra.AstraError):
        P.filter_taps(P.FilterSpec('projection', custom=spec1[:-1]), n)
    with pytest.raises(astra.AstraError):
        P.filter_taps(P.FilterSpec('sinogram', custom=specs[:-1]), n, views)


def test_filter_names(astra):
    P = importlib.import_module("astra-toolbox_b200.projector")
    assert P.filter_code('Ram-Lak') == 1 and P.filter_code('ramlak') == 1
    assert P.filter_code('rsinogram') == 21 and P.filter_code('none') == 0
    with pytest.raises(astra.AstraError):
        P.filter_code('shepp-logan-typo')
