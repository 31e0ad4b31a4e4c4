"""Film post-step against the oracle: sample variance, tone-mapped LDR blits (8-bit and float)
for every tone mapper, and the frame error against the power-of-two checkpoint.

The small scene is rendered as five one-sample frames (the reference's Device::render unit), so
the checkpoint is the image after 4 samples. Both sides accumulate the same samples, but a
5-sample image keeps each path's few-ulp differences (and the odd near-tie hit), so the bars are
per-pixel fractions:
  * HDR: >= 99% of values within 1e-3 relative; variance: >= 98% within 1e-2 relative;
  * 8-bit LDR: >= 98% of pixels within one step per channel;
  * float LDR: >= 99% of values within 1e-3;
  * frame error: relative 1e-2.
"""
import numpy as np
import pytest

import prt_scenes
import prt_types as T

pytestmark = pytest.mark.gpu

TONES = [(0, 1.0, 0.0), (1, 1.5, 0.0), (2, 1.0, 0.3), (3, 1.2, 0.0), (4, 0.8, 0.0), (5, 2.0, 0.0)]


@pytest.fixture(scope="module")
def film(device):
    s = prt_scenes.cornell(seed=0, width=64, height=64, spp=1)
    device.setup(s, seed=0, aov_mask=T.PRT_AOV_HDR_VAR)
    device.clear_frame()
    for _ in range(5):
        device.render(1)
    yield device
    device.tone_mapper(T.PRT_TONE_NONE)


def test_variance_matches(film, golden):
    z = golden("film.npz")
    hdr = film.blit_frame(T.PRT_BLIT_HDR)
    assert np.mean(np.isclose(hdr, z["hdr"], rtol=1e-3, atol=1e-6)) >= 0.99
    var = film.blit_frame(T.PRT_BLIT_HDR_VAR)
    assert np.mean(np.isclose(var, z["var"], rtol=1e-2, atol=1e-6)) >= 0.98


@pytest.mark.parametrize("kind,exposure,burn", TONES, ids=["none", "linear", "reinhard", "aces", "filmic", "log"])
def test_tone_mapped_blits_and_error(film, golden, kind, exposure, burn):
    z = golden("film.npz")
    film.tone_mapper(kind, exposure, burn)
    ldr = film.blit_frame(T.PRT_BLIT_LDR)
    ref = z[f"ldr{kind}"]
    chans = lambda a: np.stack([(a >> 16) & 255, (a >> 8) & 255, a & 255], -1).astype(np.int32)
    d = np.abs(chans(ldr) - chans(ref))
    assert np.mean(d.max(-1) <= 1) >= 0.98
    rgb = film.blit_frame(T.PRT_BLIT_LDR_RGB)
    assert np.mean(np.abs(rgb - z[f"ldrrgb{kind}"]) <= 1e-3) >= 0.99
    err = film.frame_error()
    assert abs(err / float(z[f"error{kind}"]) - 1.0) < 1e-2, (err, float(z[f"error{kind}"]))


def test_film_rejects_variance_without_the_aov(device):
    s = prt_scenes.cornell(seed=0, width=64, height=64, spp=1)
    device.setup(s, seed=0)
    device.render(1)
    with pytest.raises(ValueError):
        device.blit_frame(T.PRT_BLIT_HDR_VAR)
