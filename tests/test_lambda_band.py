"""The uniform-band wavelength policy (FTB_LAMBDA_UNIFORM_380_780; no counterpart in the
reference, whose emission always draws lambda from the emitter's SPD): lambda = 380 + 400 u
from the photon's own variate, the carried power times pdf_SPD(lambda) * 400 nm.  The oracle
restates it; here it is checked against the same arithmetic written out in Python from the
photons' random streams, photon by photon, through the energy it books at emission."""
import numpy as np
import pytest

import cases
from goodphotons_b200 import abi, scenes


def band_weights(desc, oracle, first, n):
    """Per-photon (lambda, weight) of the band policy for the one quad emitter of `desc`:
    its lambda variate is the photon's 5th uniform (2 for the point, 2 for the cosine
    direction, then lambda)."""
    em = desc.emitters[0]
    cdf = desc.emitter_cdf[em.cdf_offset: em.cdf_offset + em.cdf_n + 1]
    lam, wts = [], []
    for k in range(first, first + n):
        u = oracle.uniforms(k, 5)[4]
        l = 380.0 + 400.0 * u
        b = min(max(int((l - 360.0) / em.step), 0), em.cdf_n - 1)
        lam.append(l)
        wts.append((cdf[b + 1] - cdf[b]) / em.step * 400.0)
    return np.array(lam), np.array(wts)


def test_emitted_energy_is_the_band_weighted_power(L, oracle):
    """With no bounces the emitted tally is the sum of the photons' power x weight, in photon
    order (one thread), bit for bit."""
    desc = scenes.make_cornell(L)
    cam = cases.camera(L, 32)
    n, first = 2000, 12345
    out = oracle.trace(desc, cam, n, seed_base=first, max_bounce=0, threads=1, lambda_mode=abi.LAMBDA_UNIFORM_380_780)
    lam, wts = band_weights(desc, oracle, first, n)
    assert lam.min() >= 380.0 and lam.max() < 780.0
    power = desc.emitters[0].power
    expect = 0.0
    for w in wts:
        if w > 0.0:
            expect += power * 1.0 * w
    assert out["energy"][0] == expect


def test_band_policy_changes_only_the_wavelength_draw(L, oracle):
    """Same photons, same geometry decisions before the wavelength matters: on a scene with
    achromatic walls the hit sequences do not depend on the policy, and the band's mean
    weight is the SPD's share of 380-780 nm (to Monte Carlo precision)."""
    desc = scenes.make_cornell(L)
    cam = cases.camera(L, 32)
    n = 4096
    a = oracle.trace(desc, cam, n, seed_base=7, max_bounce=8, threads=2, logs=True)
    b = oracle.trace(desc, cam, n, seed_base=7, max_bounce=8, threads=2, logs=True,
                     lambda_mode=abi.LAMBDA_UNIFORM_380_780)
    assert (a["logs"]["n_hits"] > 0).any()
    em = desc.emitters[0]
    cdf = desc.emitter_cdf[em.cdf_offset: em.cdf_offset + em.cdf_n + 1]
    share = cdf[int(round((780.0 - 360.0) / em.step))] - cdf[int(round((380.0 - 360.0) / em.step))]
    _, wts = band_weights(desc, oracle, 7, n)
    assert abs(wts.mean() - share) < 4 * wts.std() / np.sqrt(n)
    # the first hit is decided before any spectral quantity: identical under both policies
    first_a = a["logs"]["prims"][:, 0]
    first_b = b["logs"]["prims"][:, 0]
    np.testing.assert_array_equal(first_a, first_b)


def test_hero_bundle_band_weights(L, oracle):
    """Hero bundles under the band policy: C wavelengths from one variate, stratified as
    hero.h:100-113 does (u + i/C wrapped into [0, 1)), each carrying power/C times its own
    band weight; with no bounces the emitted tally is their sum, photon by photon."""
    desc = scenes.make_cornell(L)
    cam = cases.camera(L, 32)
    n, first, C = 1000, 999, 4
    out = oracle.trace(desc, cam, n, seed_base=first, max_bounce=0, threads=1, hero_c=C,
                       lambda_mode=abi.LAMBDA_UNIFORM_380_780)
    em = desc.emitters[0]
    cdf = desc.emitter_cdf[em.cdf_offset: em.cdf_offset + em.cdf_n + 1]

    def weight(u):
        lam = 380.0 + 400.0 * u
        b = min(max(int((lam - 360.0) / em.step), 0), em.cdf_n - 1)
        return (cdf[b + 1] - cdf[b]) / em.step * 400.0

    expect = 0.0
    for k in range(first, first + n):
        u = oracle.uniforms(k, 5)[4]
        w = [weight(u)]
        for i in range(1, C):
            uu = u + i / C
            if uu >= 1.0:
                uu -= 1.0
            w.append(weight(uu))
        if not w[0] > 0.0:
            continue
        s = 0.0
        for wi in w:
            s += em.power * 1.0 / C * wi
        expect += s
    assert out["energy"][0] == expect


@pytest.mark.parametrize("hero", [1, 4])
def test_band_policy_conserves_energy(L, oracle, hero):
    """Under the band policy every photon's weight flows through its path like the power it
    replaces: absorbed + sensor + escaped + residual equals emitted (EnergyReport's
    sum/emitted == 1 check, main.cpp:13693-13696) -- photon by photon for one wavelength;
    for bundles only in expectation, as under the SPD policy, because a dielectric drops the
    secondary wavelengths and scales the hero by C (hero.h:28-70)."""
    desc = scenes.make_glass(L, level=2)
    cam = cases.camera(L, 32)
    out = oracle.trace(desc, cam, 20_000, seed_base=3, max_bounce=16, threads=2, hero_c=hero,
                       lambda_mode=abi.LAMBDA_UNIFORM_380_780)
    emitted, absorbed, sensor, escaped, residual = out["energy"]
    assert emitted > 0
    tol = 1e-9 if hero == 1 else 1e-2
    assert abs(absorbed + sensor + escaped + residual - emitted) <= tol * emitted
