"""BSDF parity: the device's Standard-material BSDFs against the reference's own
(Material::getBsdf + BsdfSimd::eval/sample compiled from its sources), on seeded
(wo, wi, sample) tuples in a canonical shading context, one case per lobe combination.

Agreement is limited by the reference's SIMD numerics: its reciprocals and square-root
reciprocals are rcpps/rsqrtps plus one Newton step (~1e-7 relative error), which peaky
low-roughness GGX lobes and the (1 - E) energy-compensation factors amplify, and sampling makes
discrete choices (lobe, reflect/refract) that flip when a sample lands within that error of a
threshold. The bar per case: >= 99.9% of evaluations within 1e-5 relative (1e-6 absolute
floor), >= 99.99% within 1e-3; >= 98% of samples within 1e-5 and >= 99.9% within 1e-3; the BSDF
flags always equal.
"""
import numpy as np
import pytest

import bsdf_cases

pytestmark = pytest.mark.gpu

CASES = bsdf_cases.cases()


def check(gpu, ref):
    tight = bsdf_cases.compare(gpu, ref, rel=1e-5)
    loose = bsdf_cases.compare(gpu, ref, rel=1e-3)
    assert tight["flags"].all()
    assert tight["eval"].mean() >= 0.999, 1 - tight["eval"].mean()
    assert loose["eval"].mean() >= 0.9999, 1 - loose["eval"].mean()
    assert tight["sample"].mean() >= 0.98, 1 - tight["sample"].mean()
    assert loose["sample"].mean() >= 0.999, 1 - loose["sample"].mean()


@pytest.mark.parametrize("name,material,medium", CASES, ids=[c[0] for c in CASES])
def test_bsdf_matches_fixture(device, golden, name, material, medium):
    """Against the committed oracle outputs (512 tuples per case)."""
    z = golden("bsdf.npz")
    tup = bsdf_cases.tuples(512, 1)
    gpu = device.bsdf_query(material, tup, medium)
    ref = z[name]
    tight = bsdf_cases.compare(gpu, ref, rel=1e-5)
    loose = bsdf_cases.compare(gpu, ref, rel=1e-3)
    assert tight["flags"].all()
    assert loose["eval"].mean() >= 0.998 and loose["sample"].mean() >= 0.99


@pytest.mark.parametrize("name,material,medium", CASES, ids=[c[0] for c in CASES])
def test_bsdf_million_tuples(device, name, material, medium):
    """1M seeded tuples per case against the live oracle (skipped where it is not built)."""
    ref_mod = pytest.importorskip("ref")
    if not ref_mod.ref_available():
        pytest.skip("oracle/_ref not built")
    tup = bsdf_cases.tuples(1 << 20, 2)
    check(device.bsdf_query(material, tup, medium), ref_mod.bsdf_query(material, tup, medium))


# Layout of prt_cuda_albedo_tables (bsdf/albedo_tables.cpp:95-130): 3D tables are
# [roughness][eta][cosThetaO] of 16 each, 2D averages [roughness][eta].
TABLES = [("ggx_dir", (32, 32), None), ("ggx_avg", (32,), None),
          ("diel_eta_dir", (16, 16, 16), 15), ("diel_eta_avg", (16, 16), 15),
          ("diel_rcp_dir", (16, 16, 16), 0), ("diel_rcp_avg", (16, 16), 0),
          ("refl_dir", (16, 16, 16), 15), ("refl_avg", (16, 16), 15),
          ("sheen_dir", (16, 16), None)]


def test_albedo_tables_match_the_reference(device):
    """Energy-compensation tables against the reference's precomputeAlbedoTables, entry by entry:
    GGX (directional and average), dielectric with eta in [1/3, 1] and in [1, 3], dielectric
    reflection, sheen, all within 2e-5 -- except the eta = 1 slices (index 15 of the [1/3, 1]
    tables, index 0 of the [1, 3] tables). There the integrand degenerates (the refracted half
    vector is undefined when the two sides' indices match), and the reference's eta is its
    approximate reciprocal rcp(1) = 0.99999994 on AVX2 rather than 1, so those entries depend on
    the CPU; they are checked to be finite albedos in [0, 1]. The reflection-EC and
    artistic-conductor-EC tables serve only the reference's specular-albedo AOV and are not part
    of this path."""
    import ref

    got = device.albedo_tables()
    want = ref.albedo_tables()
    assert got.shape == want.shape
    o = 0
    for name, shape, eta1 in TABLES:
        n = int(np.prod(shape))
        a = got[o:o + n].reshape(shape)
        b = want[o:o + n].reshape(shape)
        o += n
        keep = np.ones(shape, bool)
        if eta1 is not None:
            keep[:, eta1] = False
            g1 = a[:, eta1]
            assert np.isfinite(g1).all() and (g1 >= 0).all() and (g1 <= 1.0 + 1e-3).all(), name
        d = np.abs(a - b)[keep]
        assert d.max() < 2e-5, (name, d.max())
    assert o == len(want)


def microfacet_tuples(n, seed):
    """(alpha, s.x, s.y, wo) with alpha = roughnessToAlpha(roughness) for roughness in [0, 1]
    (bsdf/microfacet.h:11: max(roughness^2, 0.001)) and wo in the upper hemisphere."""
    rng = np.random.default_rng(seed)
    alpha = np.maximum(rng.uniform(0.0, 1.0, n) ** 2, 0.001)
    s = rng.uniform(0.0, 1.0, (n, 2))
    wo = rng.normal(size=(n, 3))
    wo[:, 2] = np.abs(wo[:, 2]) + 1e-3
    wo /= np.linalg.norm(wo, axis=1, keepdims=True)
    return np.concatenate([alpha[:, None], s, wo], 1).astype(np.float32)


@pytest.mark.parametrize("dist", ["beckmann", "ggx_visible"])
def test_microfacet_sampling_matches_the_reference(device, dist):
    """BeckmannDistribution::sample (bsdf/beckmann_distribution.h:21-42, the distribution of the
    reference's CarPaint flakes) and GGXDistribution::sampleVisible (bsdf/ggx_distribution.h:52-82)
    on 1M seeded tuples, against the reference's scalar instantiation (the scalar library's log,
    sqrt and sincos): sampled normal and pdf within 1e-5 relative for >= 99.99% of tuples and within
    1e-3 for all. Against the SIMD instantiation (its own polynomial log and approximate reciprocal
    square root; its sampled normals differ from its own scalar instantiation's by up to 1.4e-4)
    the bar is the one the BSDF cases use for samples."""
    import ref

    kind = {"beckmann": 1, "ggx_visible": 2}[dist]
    tup = microfacet_tuples(1 << 20, 5)
    gpu = device.microfacet_query(kind, tup).astype(np.float64)

    def within(ref_out, rel):
        r = ref_out.astype(np.float64)
        m_ok = np.abs(gpu[:, 0:3] - r[:, 0:3]) <= np.maximum(rel, 2e-6)
        p_ok = np.abs(gpu[:, 3] - r[:, 3]) <= rel * np.maximum(np.abs(gpu[:, 3]), np.abs(r[:, 3])) + 1e-6
        return m_ok.all(1) & p_ok

    scalar = ref.microfacet_query(kind, tup, simd=False)
    assert within(scalar, 1e-5).mean() >= 0.9999, 1 - within(scalar, 1e-5).mean()
    assert within(scalar, 1e-3).all()
    simd = ref.microfacet_query(kind, tup, simd=True)
    assert within(simd, 1e-5).mean() >= 0.98 and within(simd, 1e-3).mean() >= 0.999
