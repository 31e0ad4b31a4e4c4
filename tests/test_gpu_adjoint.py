"""Path-replay adjoint (prt_cuda_adjoint) against finite differences and a closed form.

The adjoint is wrapped in a torch.autograd.Function here, in the test harness only:
forward = render (frame form), backward = prt_cuda_adjoint with dLoss/dImage.

Checks:
  * a Lambertian plane under a distant light, whose pixels are albedo * K with K in closed form
    (sun radiance * sin^2(half angle) * cos(sun zenith)): the gradient of an L2 loss w.r.t. the
    albedo texel matches 2 * sum((albedo K - target) K) within 1%;
  * the same plane, exactly: the renderer is linear in the albedo, so the adjoint equals
    sum(dL/dI * I(albedo = 1)) at the same samples (relative 1e-4);
  * the inverse-rendering scene (textured floor and back wall, rough specular spheres):
    cosine similarity >= 0.99 between the adjoint gradient and central finite differences
    (h = 1e-3, common random numbers: the same sampler seed and samples, 4096 spp) on 32
    randomly chosen parameters (texel channels and sphere roughnesses).
"""
import math

import numpy as np
import pytest

import prt_cuda
import prt_scenes
import prt_types as T

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


class RenderImage(torch.autograd.Function):
    """image = render(texture values, roughness values); backward = path-replay adjoint."""

    @staticmethod
    def forward(ctx, textures, roughness, dev, scene, params, spp, seed):
        push_params(dev, scene, params, textures, roughness)
        dev.init_sampler(seed)
        dev.clear_frame()
        dev.render(spp)
        img = torch.empty((scene.height, scene.width, 3), dtype=torch.float32, device="cuda")
        dev.blit_frame(out=img)
        torch.cuda.synchronize()
        ctx.dev, ctx.scene, ctx.params, ctx.spp = dev, scene, params, spp
        return img

    @staticmethod
    def backward(ctx, grad_img):
        dev, scene, params = ctx.dev, ctx.scene, ctx.params
        n_tex = sum(int(t.size) for t in scene.textures)
        gt = torch.zeros(max(n_tex, 1), dtype=torch.float32, device="cuda")
        gr = torch.zeros(len(scene.materials), dtype=torch.float32, device="cuda")
        dev.adjoint(grad_img.contiguous(), ctx.spp, first_sample=0, grad_textures=gt, grad_roughness=gr)
        tex_grad = torch.cat([gt[tex_slice(scene, t)] for t in params["textures"]]) if params["textures"] else None
        rough_grad = gr[params["roughness"]] if params["roughness"] else None
        return tex_grad, rough_grad, None, None, None, None, None


def tex_slice(scene, t):
    start = sum(int(x.size) for x in scene.textures[:t])
    return slice(start, start + int(scene.textures[t].size))


def push_params(dev, scene, params, textures, roughness):
    """Writes flat parameter vectors into the device scene (textures row 0 at the top)."""
    off = 0
    for t in params["textures"]:
        n = int(scene.textures[t].size)
        dev.update_texture(t, textures[off:off + n].detach().contiguous())
        off += n
    for k, m in enumerate(params["roughness"]):
        mat = scene.materials[m]
        mat.specular_roughness = float(roughness[k])
        dev.update_material(m, mat)


def flat_params(scene, params):
    tex = torch.cat([torch.from_numpy(scene.textures[t]).reshape(-1) for t in params["textures"]]).cuda()
    rough = torch.tensor([scene.materials[m].specular_roughness for m in params["roughness"]],
                         dtype=torch.float32, device="cuda")
    return tex, rough


@pytest.fixture(scope="module")
def dev():
    d = prt_cuda.DeviceCuda(0)
    yield d
    d.close()


def render_np(dev, spp, seed):
    dev.init_sampler(seed)
    dev.clear_frame()
    dev.render(spp)
    return dev.blit_frame().astype(np.float64)


def test_plane_gradient_matches_closed_form(dev):
    scene, k = prt_scenes.lit_plane(albedo=(0.5, 0.5, 0.5), spp=256)
    dev.setup(scene, seed=0)
    params = {"textures": [0], "roughness": []}
    rho_t = np.array([0.2, 0.5, 0.7])
    target = torch.tensor(rho_t * k, dtype=torch.float32, device="cuda").expand(scene.height, scene.width, 3)
    tex, _ = flat_params(scene, params)
    tex.requires_grad_(True)
    img = RenderImage.apply(tex, None, dev, scene, params, scene.spp, 0)
    loss = ((img - target) ** 2).sum()
    loss.backward()
    got = tex.grad.cpu().numpy().reshape(3)
    n = scene.width * scene.height
    want = 2.0 * n * (0.5 - rho_t) * k * k
    # Channel 1 has a zero-residual target: compare against the scale of the others.
    scale = np.abs(want).max()
    assert np.all(np.abs(got - want) <= 0.01 * scale), (got, want)
    # The rendered image itself matches the closed form.
    assert abs(float(img.detach().mean()) / (0.5 * k) - 1.0) < 0.01


def test_plane_adjoint_is_exact_for_a_linear_renderer(dev):
    scene, k = prt_scenes.lit_plane(albedo=(0.3, 0.6, 0.9), spp=32)
    dev.setup(scene, seed=4)
    img = render_np(dev, scene.spp, 4)
    dev.update_texture(0, np.ones((1, 1, 3), np.float32))
    unit = render_np(dev, scene.spp, 4)                      # I(albedo = 1), same samples
    dev.update_texture(0, np.array([0.3, 0.6, 0.9], np.float32).reshape(1, 1, 3))
    rng = np.random.default_rng(1)
    dl = rng.normal(size=img.shape).astype(np.float32)
    gt, _, _ = dev.adjoint(dl, scene.spp, first_sample=0)
    want = (dl.astype(np.float64) * unit).reshape(-1, 3).sum(0)
    assert np.allclose(gt[:3], want, rtol=1e-4, atol=1e-6 * np.abs(want).max()), (gt[:3], want)


def loss_np(img, target):
    return float(((img - target) ** 2).sum())


def test_inverse_scene_gradient_matches_finite_differences(dev):
    spp_fd, h = 4096, 1e-3
    target_scene, _ = prt_scenes.cornell_inverse(seed=0, target=True, spp=64)
    dev.setup(target_scene, seed=7)
    target = render_np(dev, 64, 7)
    scene, params = prt_scenes.cornell_inverse(seed=0, target=False)
    dev.setup(scene, seed=0)
    base = render_np(dev, spp_fd, 0)
    # Adjoint at the same samples.
    dl = (2.0 * (base - target)).astype(np.float32)
    gt, gr, st = dev.adjoint(dl, spp_fd, first_sample=0)
    # 32 random parameters: 24 texel channels (floor and back wall), 8 sphere roughnesses.
    rng = np.random.default_rng(3)
    size = scene.textures[0].shape[0]
    picks = []
    for _ in range(24):
        t = int(rng.integers(0, 2))
        y, x, c = int(rng.integers(0, size)), int(rng.integers(0, size)), int(rng.integers(0, 3))
        picks.append(("tex", t, (y, x, c)))
    for m in rng.choice(params["roughness"], 8, replace=False):
        picks.append(("rough", int(m), None))
    adj, fd = [], []
    for kind, idx, where in picks:
        if kind == "tex":
            y, x, c = where
            tex = scene.textures[idx]
            v0 = float(tex[y, x, c])
            vals = []
            for sgn in (1, -1):
                tex[y, x, c] = v0 + sgn * h
                dev.update_texture(idx, tex)
                vals.append(loss_np(render_np(dev, spp_fd, 0), target))
            tex[y, x, c] = v0
            dev.update_texture(idx, tex)
            adj.append(float(gt[tex_slice(scene, idx)].reshape(tex.shape)[y, x, c]))
        else:
            mat = scene.materials[idx]
            r0 = mat.specular_roughness
            vals = []
            for sgn in (1, -1):
                mat.specular_roughness = r0 + sgn * h
                dev.update_material(idx, mat)
                vals.append(loss_np(render_np(dev, spp_fd, 0), target))
            mat.specular_roughness = r0
            dev.update_material(idx, mat)
            adj.append(float(gr[idx]))
        fd.append((vals[0] - vals[1]) / (2 * h))
    adj, fd = np.array(adj), np.array(fd)
    cos = float(adj @ fd / (np.linalg.norm(adj) * np.linalg.norm(fd)))
    tex_cos = float(adj[:24] @ fd[:24] / (np.linalg.norm(adj[:24]) * np.linalg.norm(fd[:24])))
    assert cos >= 0.99, (cos, tex_cos, adj, fd)
    assert tex_cos >= 0.99, (tex_cos, adj[:24], fd[:24])


def test_adjoint_rejects_unsupported_materials(dev):
    scene = prt_scenes.terrain(seed=0, grid=32, n_spheres=8, width=64, height=64, spp=1)
    dev.setup(scene, seed=0)
    with pytest.raises(ValueError):
        dev.adjoint(np.zeros((64, 64, 3), np.float32), 1)
