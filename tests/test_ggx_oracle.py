"""The oracle's GGX conductor (the glossy material of the path tracer)
against its definition in FP64 (Walter et al. 2007): sample weights equal
f cos / pdf, the BRDF is reciprocal, and a white furnace loses no more than
the masking term allows."""

import numpy as np

import oracle_lib as ol


def _unit(v):
    return v / np.linalg.norm(v)


def _ggx_f64(n, wo, wi, alpha, f0):
    a2 = alpha * alpha
    h = _unit(wo + wi)
    nh, lh = n @ h, wi @ h
    D = a2 / (np.pi * (nh * nh * (a2 - 1) + 1) ** 2)

    def g1(v):
        nv = n @ v
        return 2 * nv / (nv + np.sqrt(a2 + (1 - a2) * nv * nv))
    F = f0 + (1 - f0) * (1 - lh) ** 5
    return F * D * g1(wo) * g1(wi) / (4 * (n @ wo) * (n @ wi)), D, h


def _cases(k, seed=0):
    rng = np.random.default_rng(seed)
    for _ in range(k):
        n = _unit(rng.normal(size=3))
        wo = _unit(rng.normal(size=3))
        if n @ wo < 0.05:
            wo = _unit(wo - 2 * (n @ wo) * n + 0.1 * n)
        alpha = rng.uniform(0.05, 0.5)
        f0 = rng.uniform(0.5, 1.0, 3)
        yield n, wo, alpha, f0, rng.uniform(0, 1), rng.uniform(0, 0.999)


def test_sample_weight_is_brdf_cos_over_pdf():
    checked = 0
    for n, wo, alpha, f0, r0, r1 in _cases(400):
        ok, wi, w = ol.ggx_sample(n, wo, alpha, f0, r0, r1)
        if not ok:
            continue
        wi64 = wi.astype(np.float64)
        f, D, h = _ggx_f64(n, wo, wi64, alpha, f0)
        pdf = D * (n @ h) / (4 * (wo @ h))
        want = f * (n @ wi64) / pdf
        assert np.allclose(w, want, rtol=2e-4, atol=1e-6), (w, want)
        checked += 1
    assert checked > 300


def test_eval_matches_definition_and_is_reciprocal():
    rng = np.random.default_rng(5)
    for n, wo, alpha, f0, _, _ in _cases(200, 1):
        wi = _unit(rng.normal(size=3))
        if n @ wi < 0.05:
            wi = _unit(wi - 2 * (n @ wi) * n + 0.1 * n)
        got = ol.ggx_eval(n, wo, wi, alpha, f0)
        want, _, _ = _ggx_f64(n, wo, wi, alpha, f0)
        assert np.allclose(got, want, rtol=2e-4), (got, want)
        back = ol.ggx_eval(n, wi, wo, alpha, f0)
        assert np.allclose(got, back, rtol=2e-4)


def _albedo_normal_f64(alpha):
    """Directional albedo at normal incidence with F0 = 1 by quadrature
    over the reflected polar angle (FP64)."""
    th = np.linspace(0, np.pi / 2, 200001)[1:-1]
    dth = th[1] - th[0]
    a2 = alpha * alpha
    nh = np.cos(th / 2)
    D = a2 / (np.pi * (nh * nh * (a2 - 1) + 1) ** 2)
    ci = np.cos(th)
    g1i = 2 * ci / (ci + np.sqrt(a2 + (1 - a2) * ci * ci))
    f = D * g1i / (4 * ci)
    return float(np.sum(f * ci * np.sin(th)) * dth * 2 * np.pi)


def test_white_furnace():
    """F0 = 1: the mean sample weight is the directional albedo, at most 1,
    and at normal incidence equal to the FP64 quadrature of f cos."""
    n = np.array([0.0, 0.0, 1.0])
    for alpha in (0.05, 0.2, 0.5):
        for theta in (0.0, 0.8):
            wo = np.array([np.sin(theta), 0.0, np.cos(theta)])
            tot, m = 0.0, 64
            for i in range(m):
                for j in range(m):
                    ok, _, w = ol.ggx_sample(n, wo, alpha, np.ones(3),
                                             (i + 0.5) / m, (j + 0.5) / m)
                    tot += w[0] if ok else 0.0
            albedo = tot / (m * m)
            assert albedo <= 1.0 + 1e-3, (alpha, theta, albedo)
            if theta == 0.0:
                want = _albedo_normal_f64(alpha)
                assert abs(albedo - want) < 0.01, (alpha, albedo, want)
