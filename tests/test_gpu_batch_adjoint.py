"""Batched path-replay adjoint (prt_cuda_batch_adjoint) against the frame-form adjoint.

Every path of a batch item is the path the frame form traces for that frame, and both replay it
with the same gradient step, so the per-item gradients agree up to the order of the atomic FP32
additions: relative L2 difference <= 1e-3 and cosine >= 0.99999.
"""
import numpy as np
import pytest

import prt_cuda
import prt_scenes

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def dev():
    d = prt_cuda.DeviceCuda(0)
    yield d
    d.close()


def problems():
    out = []
    for k, (tris, size) in enumerate([(2e4, 64), (5e4, 96), (1e4, 64)]):
        s, params = prt_scenes.terrain_inverse(seed=11 + k, tris=tris, size=size, spp=4, max_depth=4, tex_size=64)
        out.append((s, params, 100 + k))
    return out


def grads_frame(dev, scene, seed, dl):
    dev.setup(scene, seed=seed)
    gt, gr, _ = dev.adjoint(dl, scene.spp, first_sample=0)
    return gt, gr


def test_batch_adjoint_matches_frame_adjoint(dev):
    probs = problems()
    rng = np.random.default_rng(5)
    dls = [rng.normal(size=(s.height, s.width, 3)).astype(np.float32) for s, _, _ in probs]
    batch = prt_cuda.Batch(dev, [(s, seed, 0) for s, _, seed in probs])
    batch.enable_adjoint()
    batch.render()
    gts = [torch.zeros(sum(int(t.size) for t in s.textures), device="cuda") for s, _, _ in probs]
    grs = [torch.zeros(len(s.materials), device="cuda") for s, _, _ in probs]
    batch.adjoint([torch.from_numpy(d).cuda() for d in dls], gts, grs)
    for k, (s, params, seed) in enumerate(probs):
        ft, fr = grads_frame(dev, s, seed, dls[k])
        bt, br = gts[k].cpu().numpy(), grs[k].cpu().numpy()
        for a, b in ((bt, ft), (br, fr)):
            a64, b64 = a.astype(np.float64), b.astype(np.float64)
            assert np.linalg.norm(b64) > 0
            assert np.linalg.norm(a64 - b64) <= 1e-3 * np.linalg.norm(b64), (k, np.linalg.norm(a64 - b64))
            assert a64 @ b64 / (np.linalg.norm(a64) * np.linalg.norm(b64)) >= 0.99999
    batch.close()


def test_batch_adjoint_needs_enable_and_render(dev):
    probs = problems()[:1]
    s, _, seed = probs[0]
    batch = prt_cuda.Batch(dev, [(s, seed, 0)])
    dl = [torch.zeros((s.height, s.width, 3), device="cuda")]
    gt = [torch.zeros(sum(int(t.size) for t in s.textures), device="cuda")]
    gr = [torch.zeros(len(s.materials), device="cuda")]
    with pytest.raises(RuntimeError):
        batch.adjoint(dl, gt, gr)
    batch.close()


def test_batch_parameter_updates_change_the_image(dev):
    s, params, seed = problems()[0]
    batch = prt_cuda.Batch(dev, [(s, seed, 0)])
    batch.render()
    before = batch.blit(0)
    batch.update_texture(0, params["textures"][0], np.full(s.textures[0].shape, 0.9, np.float32))
    batch.render()
    after = batch.blit(0)
    assert after.mean() > before.mean()
    batch.close()
