"""Serving-form materials on the host: the oracle's OpenPBR-subset BSDF restatement against the reference's own
render/bsdf.h (fixture tests/golden/bsdf.npz made by its code): f, pdf, sampled directions, weights and success flags,
with the glossy-diffuse energy compensation off and on."""
import numpy as np

from conftest import golden


def close(a, b, rel=2e-5, abs_=1e-6):
    return np.all(np.abs(a - b) <= abs_ + rel * np.maximum(np.abs(a), np.abs(b)))


def test_oracle_bsdf_eval_matches_reference(oracle):
    g = golden("bsdf.npz")
    for gd in (0, 1):
        f, pdf = oracle.bsdf_eval(g["mats"], g["mat"], g["wo"], g["wi"], g["eta"], gd, g["ux"])
        assert close(f, g[f"f{gd}"]) and close(pdf, g[f"pdf{gd}"]), gd
        assert (g[f"pdf{gd}"] > 0).mean() > 0.3   # the cases exercise the lobes


def test_oracle_bsdf_sample_matches_reference(oracle):
    g = golden("bsdf.npz")
    for gd in (0, 1):
        wi, w, pdf, ok = oracle.bsdf_sample(g["mats"], g["mat"], g["wo"], g["eta"], gd, g["ux"], g["uvw"])
        same = ok == g[f"s_ok{gd}"]
        assert same.mean() >= 0.999, gd   # a success decision may flip only at a rounding boundary
        k = same & (ok == 1)
        assert close(wi[k], g[f"s_wi{gd}"][k], rel=1e-4, abs_=1e-5) and close(w[k], g[f"s_w{gd}"][k], rel=1e-4, abs_=1e-5)
        assert close(pdf[k], g[f"s_pdf{gd}"][k], rel=1e-4, abs_=1e-5)
        assert (g[f"s_pdf{gd}"] == 0).any() and (g[f"s_ok{gd}"] == 1).mean() > 0.5   # delta and glossy samples both present


def test_bsdf_reciprocity_and_energy(oracle):
    """Sanity of the restated lobes: non-negative f and pdf; the sampled weight of a single-lobe Lambertian material is
    its albedo."""
    g = golden("bsdf.npz")
    f, pdf = oracle.bsdf_eval(g["mats"], g["mat"], g["wo"], g["wi"], g["eta"], 1, g["ux"])
    assert np.all(f >= 0) and np.all(pdf >= 0)
    lam = np.where(g["mat"] % 8 == 0)[0]
    wi, w, p, ok = oracle.bsdf_sample(g["mats"], g["mat"][lam], g["wo"][lam], g["eta"][lam], 0, g["ux"][lam], g["uvw"][lam])
    assert np.allclose(w[ok == 1], g["mats"][g["mat"][lam][ok == 1], 0:3], rtol=1e-5)


def test_oracle_bump_terminator_matches_reference(oracle):
    """The bump-terminator term of the diffuse lobe (render/bsdf.h:67-75) with an unperturbed normal per case
    (fixture tests/golden/bsdf_bump.npz, the reference's bsdfEval / bsdfSample with nr): eval and sample agree as
    without the term; cases with nr = +z give the plain values; the term only ever darkens the diffuse lobe."""
    g, b = golden("bsdf.npz"), golden("bsdf_bump.npz")
    n = len(b["nr"])
    for gd in (0, 1):
        f, pdf = oracle.bsdf_eval(g["mats"], g["mat"], g["wo"], g["wi"], g["eta"], gd, g["ux"], nr=b["nr"])
        assert close(f, b[f"f{gd}"]) and close(pdf, b[f"pdf{gd}"]), gd
        assert np.array_equal(b[f"f{gd}"][3 * n // 4:], g[f"f{gd}"][3 * n // 4:])
        assert np.all(b[f"f{gd}"] <= g[f"f{gd}"] + 1e-7) and (b[f"f{gd}"] < g[f"f{gd}"]).mean() > 0.1
        wi, w, pdf, ok = oracle.bsdf_sample(g["mats"], g["mat"], g["wo"], g["eta"], gd, g["ux"], g["uvw"], nr=b["nr"])
        same = ok == b[f"s_ok{gd}"]
        assert same.mean() >= 0.999, gd
        k = same & (ok == 1)
        assert close(wi[k], b[f"s_wi{gd}"][k], rel=1e-4, abs_=1e-5) and close(w[k], b[f"s_w{gd}"][k], rel=1e-4, abs_=1e-5)
