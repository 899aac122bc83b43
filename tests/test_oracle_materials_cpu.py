"""Known-answer tests of the oracle's two materials without a reference
counterpart (CPU only).

The rough dielectric follows Walter, Marschner, Li and Torrance 2007,
"Microfacet models for refraction through rough surfaces"; the coat is a
diffuse base under the reference's GGX lobe (dMaterial.cu:266-288) with a
Fresnel f0 from the coat's IOR.  The oracle (oracle/ffo_render.c) restates
both as the product computes them, in FP32.  Here they are checked against
an independent float64 statement of the published formulas (different
algebraic forms: Fresnel through s- and p-polarised reflectances and Snell's
law, D through tan^2 theta), against each other (the sampler against the
pdf, by quadrature over the sphere and by Monte Carlo), and against closed
forms (normal-incidence reflectance, the smooth limit).
"""
from __future__ import annotations

import math

import numpy as np
import pytest


def _unit(v):
    v = np.asarray(v, np.float64)
    return v / np.linalg.norm(v)


def fresnel_sp(cos_i: float, eta_i: float, eta_t: float) -> float:
    """Unpolarised reflectance from Snell's law and the s/p amplitudes."""
    sin_t2 = (eta_i / eta_t) ** 2 * max(0.0, 1.0 - cos_i * cos_i)
    if sin_t2 >= 1.0:
        return 1.0
    cos_t = math.sqrt(1.0 - sin_t2)
    rs = (eta_i * cos_i - eta_t * cos_t) / (eta_i * cos_i + eta_t * cos_t)
    rp = (eta_t * cos_i - eta_i * cos_t) / (eta_t * cos_i + eta_i * cos_t)
    return 0.5 * (rs * rs + rp * rp)


def walter(n, wo, wi, alpha, eta_o, eta_t, tint):
    """f (rgb) and pdf of the rough dielectric, float64, from the paper."""
    n, wo, wi = _unit(n), _unit(wo), _unit(wi)
    co, ci = float(n @ wo), float(n @ wi)
    zero = (np.zeros(3), 0.0)
    if co <= 0 or ci == 0:
        return zero
    refl = ci > 0
    h = wo + wi if refl else eta_o * wo + eta_t * wi
    h = _unit(h)
    if h @ n < 0:
        h = -h
    woh, wih, ch = float(wo @ h), float(wi @ h), float(n @ h)
    if woh <= 0 or (refl and wih <= 0) or (not refl and wih >= 0):
        return zero
    tan2h = (1 - ch * ch) / (ch * ch)
    D = alpha ** 2 / (math.pi * ch ** 4 * (alpha ** 2 + tan2h) ** 2)

    def g1(v, vh):
        vn = float(n @ v)
        if vh / vn <= 0:
            return 0.0
        t2 = (1 - vn * vn) / (vn * vn)
        return 2.0 / (1.0 + math.sqrt(1.0 + alpha * alpha * t2))
    G = g1(wo, woh) * g1(wi, wih)
    F = fresnel_sp(woh, eta_o, eta_t)
    walter.last_F = F
    walter.last_g2 = (eta_t / eta_o) ** 2 - 1 + woh * woh   # g^2 of the Fresnel term, 0 at the critical angle
    if refl:
        f = F * D * G / (4 * abs(ci) * co)
        return np.full(3, f), F * D * ch / (4 * woh)
    den = eta_o * woh + eta_t * wih
    f = (1 - F) * D * G * abs(wih) * woh * eta_o ** 2 / (abs(ci) * co * den * den)
    pdf = (1 - F) * D * ch * eta_t ** 2 * abs(wih) / (den * den)
    return np.asarray(tint, np.float64) * f, pdf


def _random_dirs(rng, k):
    v = rng.normal(size=(k, 3))
    return v / np.linalg.norm(v, axis=1, keepdims=True)


def test_fresnel_dielectric_known_answers(oracle):
    # normal incidence: ((n - 1) / (n + 1))^2
    for n in (1.33, 1.5, 2.4):
        assert oracle.fresnel_dielectric(1.0, n) == pytest.approx(((n - 1) / (n + 1)) ** 2, rel=1e-6)
        assert oracle.fresnel_dielectric(1.0, 1.0 / n) == pytest.approx(((n - 1) / (n + 1)) ** 2, rel=1e-6)
    # total internal reflection beyond the critical angle (glass to air)
    crit = math.sqrt(1 - (1 / 1.5) ** 2)
    assert oracle.fresnel_dielectric(crit * 0.99, 1 / 1.5) == 1.0
    # grazing incidence reflects everything
    assert oracle.fresnel_dielectric(1e-6, 1.5) == pytest.approx(1.0, abs=1e-4)
    # every angle and both directions against the s/p form
    for c in np.linspace(0.01, 1.0, 60):
        for eta_o, eta_t in ((1.0, 1.5), (1.5, 1.0), (1.0, 1.33)):
            got = oracle.fresnel_dielectric(float(c), eta_t / eta_o)
            assert got == pytest.approx(fresnel_sp(float(c), eta_o, eta_t), abs=2e-6), (c, eta_o, eta_t)


@pytest.mark.parametrize("back", [0, 1])
def test_dielectric_eval_against_the_paper(oracle, back):
    rng = np.random.default_rng(7 + back)
    tint = (0.9, 0.8, 0.7)
    checked = {"refl": 0, "trans": 0}
    for _ in range(3000):
        n = _unit(rng.normal(size=3))
        wo = _unit(rng.normal(size=3))
        if wo @ n < 0:
            wo = -wo
        wi = _unit(rng.normal(size=3))
        r = float(rng.uniform(0.2, 0.9))
        ior = 1.5
        eta_o, eta_t = (ior, 1.0) if back else (1.0, ior)
        f, pdf = oracle.dielectric_eval(tint, r, ior, back, n, wo, wi)
        fw, pw = walter(n, wo, wi, r * r, eta_o, eta_t, tint)
        if pw == 0.0:
            assert pdf == 0.0 and not f.any()
            continue
        trans = wi @ n < 0
        checked["trans" if trans else "refl"] += 1
        # FP32 conditioning: near the critical angle the refracted direction
        # grazes the microfacet; g^2 = n^2 - 1 + (wo.h)^2 of the Fresnel term
        # then cancels to a few ulps, and so does 1 - F
        rel = 2e-4 + (2e-7 / max(walter.last_g2, 1e-12) if trans else 0.0)
        assert pdf == pytest.approx(pw, rel=rel, abs=1e-9)
        np.testing.assert_allclose(f, fw, rtol=rel, atol=1e-9)
    assert checked["refl"] > 300 and checked["trans"] > 200


@pytest.mark.parametrize("r,back", [(0.5, 0), (0.5, 1), (0.3, 0)])
def test_dielectric_sampler_matches_its_pdf(oracle, r, back):
    """The directions the sampler draws are distributed as the pdf says:
    E[f |cos| / pdf] over samples equals the quadrature of f |cos| over the
    sphere (the directional albedo), and the quadrature of the pdf equals the
    fraction of valid samples."""
    ior = 1.5
    n = np.array([0.0, 0.0, 1.0])
    wo = _unit([0.6, 0.0, 0.8])
    rng = np.random.default_rng(11)
    m = 4000
    w_sum, valid = 0.0, 0
    for _ in range(m):
        e = rng.random(3)
        ok, wi = oracle.dielectric_sample((1, 1, 1), r, ior, back, n, wo, *map(float, e))
        if not ok:
            continue
        f, pdf = oracle.dielectric_eval((1, 1, 1), r, ior, back, n, wo, wi)
        if pdf > 0:
            valid += 1
            w_sum += f[0] * abs(wi @ n) / pdf
    mc_albedo = w_sum / m
    # quadrature over the sphere (cos theta, phi grid, both hemispheres)
    nt, nph = 300, 300
    ct = (np.arange(nt) + 0.5) / nt * 2 - 1
    ph = (np.arange(nph) + 0.5) / nph * 2 * math.pi
    dA = (2.0 / nt) * (2 * math.pi / nph)
    q_refl, q_trans, q_pdf = 0.0, 0.0, 0.0
    for c in ct:
        s = math.sqrt(1 - c * c)
        for p in ph:
            wi = np.array([s * math.cos(p), s * math.sin(p), c])
            f, pdf = oracle.dielectric_eval((1, 1, 1), r, ior, back, n, wo, wi)
            if c > 0:
                q_refl += f[0] * abs(c) * dA
            else:
                q_trans += f[0] * abs(c) * dA
            q_pdf += pdf * dA
    assert q_pdf == pytest.approx(valid / m, abs=0.02)
    assert mc_albedo == pytest.approx(q_refl + q_trans, rel=0.03)
    # no energy is created: the transmitted radiance carries the factor
    # (eta_o / eta_t)^2, so the flux albedo is refl + trans (eta_t / eta_o)^2
    eta_o, eta_t = (ior, 1.0) if back else (1.0, ior)
    assert q_refl + q_trans * (eta_t / eta_o) ** 2 < 1.0


def test_dielectric_smooth_limit(oracle):
    """At roughness 0.05 the sampled directions are the mirror and Snell
    directions of the macro surface."""
    ior = 1.5
    n = np.array([0.0, 0.0, 1.0])
    th = math.radians(40)
    wo = np.array([math.sin(th), 0.0, math.cos(th)])
    mirror = np.array([-wo[0], 0.0, wo[2]])
    sin_t = math.sin(th) / ior
    snell = np.array([-sin_t, 0.0, -math.sqrt(1 - sin_t * sin_t)])
    rng = np.random.default_rng(3)
    for _ in range(200):
        e = rng.random(3)
        ok, wi = oracle.dielectric_sample((1, 1, 1), 0.05, ior, 0, n, wo, *map(float, e))
        assert ok
        target = mirror if wi[2] > 0 else snell
        assert float(np.dot(wi, target)) > 0.995


def test_dielectric_sample_reflection_and_refraction_fractions(oracle):
    """The share of reflected samples is the mean Fresnel reflectance at the
    sampled microfacets: close to F(cos theta_o) for a nearly smooth surface."""
    ior = 1.5
    n = np.array([0.0, 0.0, 1.0])
    th = math.radians(60)
    wo = np.array([math.sin(th), 0.0, math.cos(th)])
    rng = np.random.default_rng(5)
    refl = 0
    m = 6000
    for _ in range(m):
        ok, wi = oracle.dielectric_sample((1, 1, 1), 0.1, ior, 0, n, wo, *map(float, rng.random(3)))
        refl += ok and wi[2] > 0
    assert refl / m == pytest.approx(fresnel_sp(math.cos(th), 1.0, ior), abs=0.02)


def coat_ref(albedo, r, ior, n, wi, wo):
    """The coat, float64: reference GGX lobe (alpha = r^2, Schlick-GGX G with
    k = (r+1)^2/8, Schlick F with f0 = ((ior-1)/(ior+1))^2, white, no metal)
    plus albedo (1 - F) / pi; pdf of the 50/50 continuation."""
    n, wi, wo = _unit(n), _unit(wi), _unit(wo)
    r0 = ((ior - 1) / (ior + 1)) ** 2
    h = _unit(wo + wi)
    nl, nv, nh = max(n @ wi, 0), max(n @ wo, 0), max(n @ h, 0)
    a2 = r ** 4
    D = a2 / (math.pi * (nh * nh * (a2 - 1) + 1) ** 2)
    k = (r + 1) ** 2 / 8
    G = (nl / (nl * (1 - k) + k)) * (nv / (nv * (1 - k) + k))
    F = r0 + (1 - r0) * (1 - max(h @ wi, 0)) ** 5
    spec = D * G * F / max(4 * nv * nl, 1e-3)
    f = spec + np.asarray(albedo) * (1 - F) / math.pi
    spec_pdf = D * max(h @ n, 0) / max(4 * max(wo @ h, 0), 1e-3)
    return f, 0.5 * spec_pdf + 0.5 * max(n @ wi, 0) / math.pi


def test_coat_against_its_formula(oracle):
    rng = np.random.default_rng(9)
    for _ in range(2000):
        n = _unit(rng.normal(size=3))
        wo = _unit(rng.normal(size=3))
        wi = _unit(rng.normal(size=3))
        if wo @ n < 0:
            wo = -wo
        if wi @ n < 0:
            wi = -wi
        r = float(rng.uniform(0.1, 0.9))
        alb = rng.uniform(0.1, 0.9, 3)
        f, pdf = oracle.coat_eval(alb, r, 1.5, n, wi, wo)
        fr, pr = coat_ref(alb, r, 1.5, n, wi, wo)
        np.testing.assert_allclose(f, fr, rtol=5e-4, atol=1e-6)
        assert pdf == pytest.approx(pr, rel=5e-4, abs=1e-6)


def test_oracle_refuses_unknown_kinds(oracle):
    """A material kind the oracle does not restate is an error, not a
    silent substitute."""
    from firefly_b200 import scenes
    scn = scenes.small_room(seed=0, width=8, height=8)
    scn.materials[1].kind = 7
    with pytest.raises(ValueError, match="does not restate"):
        oracle.render(scn, 8, 8, 1, max_depth=2, light=0, mode=1)
