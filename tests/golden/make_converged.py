"""Generates the full-size fixtures in tests/golden/ from the oracle (the reference's pathStream
renderer and its ray queries, compiled from its sources into oracle/_ref/libprt_ref.so).

These take CPU-minutes to CPU-hours, so they live apart from make_golden.py. Run from the
repository root, one or more of:

    python tests/golden/make_converged.py terrain_rays terrain_ties cornell terrain

Fixtures:
  terrain_rays.npz     closest hits on the full terrain scene (2.6M triangles) of three ray sets
                       chosen from the oracle's own rays: 16,384 primary rays (sample index 0,
                       random pixels), 16,384 bounce rays (from those primary hits, cosine-weighted
                       around the geometric normal, near = the reference's hit epsilon) and 16,384
                       random rays through the scene's box; plus occlusion of the bounce rays at a
                       finite far
  terrain_ties.npz     rays through shared vertices and edges of the terrain grid (several triangles hit
                       at one point) with their closest hits and the incident triangles of each target
  cornell_full.npz     the small scene at its full size (256x256, depth 5) at 4096 spp, seeds 0 and 1,
                       with the ray counts
  terrain_full.npz     the terrain scene at its full size (1920x1080, depth 8, RR from depth 3,
                       sun-sky) at SPP_TERRAIN spp: the seed-0 image (float16: the values stay far
                       below its range and its rounding is far below the noise) and the relMSE
                       between the seed-0 and seed-1 images, which is the acceptance scale
"""
import pathlib
import sys
import time

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT / "oidn-protoray_b200"))
sys.path.insert(0, str(ROOT / "oracle"))
import prt_scenes  # noqa: E402
import ref  # noqa: E402

OUT = pathlib.Path(__file__).resolve().parent
SPP_CORNELL = 4096
SPP_TERRAIN = 1024
CHUNK = 256


def rel_mse(a, b):
    a, b = a.astype(np.float64), b.astype(np.float64)
    return float(np.mean((a - b) ** 2 / (b ** 2 + 1e-2)))


def _render(scene, seed, spp, label):
    dev = ref.RefDevice(scene, seed=seed)
    rays, secs, done = 0.0, 0.0, 0
    t0 = time.time()
    while done < spp:
        n = min(CHUNK, spp - done)
        st = dev.render(n)
        rays += st["rays"]
        secs += st["seconds"]
        done += n
        print(f"{label} seed {seed}: {done}/{spp} spp, {rays / 1e6 / secs:.1f} Mrays/s, {time.time() - t0:.0f} s",
              flush=True)
    img = dev.blit()
    dev.close()
    return img, rays


def make_cornell():
    out = {}
    for seed in (0, 1):
        img, rays = _render(prt_scenes.cornell(seed=0, width=256, height=256, spp=SPP_CORNELL), seed, SPP_CORNELL,
                            "cornell")
        out[f"seed{seed}"] = img
        out[f"seed{seed}_rays"] = np.float64(rays)
    out["spp"] = np.int32(SPP_CORNELL)
    np.savez_compressed(OUT / "cornell_full.npz", **out)
    print("cornell seed-to-seed relMSE", rel_mse(out["seed1"], out["seed0"]))


def terrain_scene(spp=1):
    return prt_scenes.terrain(seed=0, spp=spp)


def make_terrain():
    imgs, rays = {}, {}
    for seed in (0, 1):
        imgs[seed], rays[seed] = _render(terrain_scene(SPP_TERRAIN), seed, SPP_TERRAIN, "terrain")
        np.save(f"/tmp/prt_terrain_full_seed{seed}.npy", imgs[seed])
    seeds = rel_mse(imgs[1], imgs[0])
    assert float(np.abs(imgs[0]).max()) < 6e4
    np.savez_compressed(OUT / "terrain_full.npz", seed0=imgs[0].astype(np.float16), seed_to_seed=np.float64(seeds),
                        seed0_rays=np.float64(rays[0]), seed1_rays=np.float64(rays[1]), spp=np.int32(SPP_TERRAIN))
    print("terrain seed-to-seed relMSE", seeds)


def _cosine_dirs(n, rng):
    """Unit vectors around +z with density cos(theta)/pi, from uniform pairs."""
    u1, u2 = rng.uniform(size=n), rng.uniform(size=n)
    r, phi = np.sqrt(u1), 2 * np.pi * u2
    return np.stack([r * np.cos(phi), r * np.sin(phi), np.sqrt(np.maximum(0.0, 1 - u1))], 1)


def make_terrain_rays(n=16384):
    s = terrain_scene()
    dev = ref.RefDevice(s, seed=0)
    rng = np.random.default_rng(2024)
    prim_rays, g, p, t = dev.query_primary(0)
    pick = rng.choice(prim_rays.shape[0], n, replace=False)
    primary = prim_rays[pick]
    out = {}
    g, p, t, u, v = dev.trace(primary)
    out.update(primary_rays=primary, primary_geom=g, primary_prim=p, primary_t=t, primary_u=u, primary_v=v)
    # Bounce rays from the primary hits (the hits of rays that missed are replaced by terrain points).
    hit = g >= 0
    o = primary[:, 0:3].astype(np.float64) + primary[:, 4:7].astype(np.float64) * t[:, None]
    miss = ~hit
    o[miss] = np.stack([rng.uniform(-45, 45, miss.sum()), np.full(miss.sum(), 12.0), rng.uniform(-45, 45, miss.sum())],
                       1)
    # Geometric normals of the hit triangles, from the scene's own arrays.
    tv = prt_scenes.tri_verts(s).reshape(-1, 3, 3).astype(np.float64)
    first = np.concatenate([[0], np.cumsum([len(m["indices"]) for m in s.meshes])])
    nrm = np.tile([0.0, 1.0, 0.0], (n, 1))
    tri = tv[np.where(hit, first[np.maximum(g, 0)] + p, 0)]
    ng = np.cross(tri[:, 1] - tri[:, 0], tri[:, 2] - tri[:, 0])
    ng /= np.linalg.norm(ng, axis=1, keepdims=True)
    ng = np.where((np.sum(ng * primary[:, 4:7], 1) > 0)[:, None], -ng, ng)
    nrm[hit] = ng[hit]
    # Frame around the normal.
    a = np.where(np.abs(nrm[:, 0:1]) > 0.9, [[0.0, 1.0, 0.0]], [[1.0, 0.0, 0.0]])
    tx = np.cross(a, nrm)
    tx /= np.linalg.norm(tx, axis=1, keepdims=True)
    ty = np.cross(nrm, tx)
    c = _cosine_dirs(n, rng)
    d = c[:, 0:1] * tx + c[:, 1:2] * ty + c[:, 2:3] * nrm
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    # The reference's hit epsilon, max(t, max|p|) * 0x1.fp-18 (core/ray.h:63-67).
    eps = np.maximum(np.where(hit, t, 0.0), np.abs(o).max(1)) * (31.0 / 16.0) * 2.0 ** -18
    far = np.full(n, 3.4028234663852886e38)
    bounce = np.concatenate([o, eps[:, None], d, far[:, None]], 1).astype(np.float32)
    g, p, t, u, v = dev.trace(bounce)
    out.update(bounce_rays=bounce, bounce_geom=g, bounce_prim=p, bounce_t=t, bounce_u=u, bounce_v=v)
    shadow = bounce.copy()
    shadow[:, 7] = rng.uniform(0.5, 40.0, n).astype(np.float32)
    out.update(shadow_rays=shadow, shadow_occ=dev.occluded(shadow))
    # Random rays through the scene's box.
    org = np.stack([rng.uniform(-50, 50, n), rng.uniform(-2, 30, n), rng.uniform(-50, 50, n)], 1)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rnd = np.concatenate([org, np.full((n, 1), 1e-4), d, np.full((n, 1), 3.4028234663852886e38)], 1).astype(np.float32)
    g, p, t, u, v = dev.trace(rnd)
    out.update(random_rays=rnd, random_geom=g, random_prim=p, random_t=t, random_u=u, random_v=v)
    dev.close()
    np.savez_compressed(OUT / "terrain_rays.npz", **out)
    print("terrain rays:", {k: int((out[k + "_geom"] >= 0).sum()) for k in ("primary", "bounce", "random")},
          "occluded", int(out["shadow_occ"].sum()))


def make_terrain_ties(n=4096, grid=1024):
    """Rays aimed at shared features of the terrain grid, where several triangles are hit at the
    same point and the closest hit is decided by the tie rule: vertical rays through interior
    vertices (six incident triangles), vertical rays through the float32 midpoints of the cells'
    diagonals (two triangles), and oblique rays toward interior vertices. For each ray the
    fixture also records how many triangles incident to the aimed-at feature there are, and the
    test counts the rays whose closest hit is one of them (the ties)."""
    s = terrain_scene()
    mesh = s.meshes[0]
    pos = mesh["positions"].astype(np.float32)
    cells = (grid - 1) * (grid - 1)
    rng = np.random.default_rng(77)
    i = rng.integers(1, grid - 1, n)
    j = rng.integers(1, grid - 1, n)

    def tri_a(ci, cj):
        return cj * (grid - 1) + ci

    def tri_b(ci, cj):
        return cells + cj * (grid - 1) + ci

    vid = j * grid + i
    incident_v = np.stack([tri_a(i, j), tri_a(i - 1, j), tri_b(i - 1, j), tri_a(i, j - 1), tri_b(i, j - 1),
                           tri_b(i - 1, j - 1)], 1)
    v = pos[vid]
    up = np.float32(20.0)
    inf = np.float32(3.4028234663852886e38)
    down = np.tile(np.array([0, -1, 0], np.float32), (n, 1))
    vert = np.concatenate([v[:, 0:1], v[:, 1:2] + up, v[:, 2:3], np.zeros((n, 1), np.float32), down,
                           np.full((n, 1), inf, np.float32)], 1).astype(np.float32)
    # Diagonal v10-v01 of cell (i, j): shared by triangles A(i, j) and B(i, j).
    ci = rng.integers(0, grid - 1, n)
    cj = rng.integers(0, grid - 1, n)
    p10 = pos[cj * grid + ci + 1]
    p01 = pos[(cj + 1) * grid + ci]
    mid = ((p10.astype(np.float64) + p01) * 0.5).astype(np.float32)
    diag = np.concatenate([mid[:, 0:1], mid[:, 1:2] + up, mid[:, 2:3], np.zeros((n, 1), np.float32), down,
                           np.full((n, 1), inf, np.float32)], 1).astype(np.float32)
    incident_d = np.stack([tri_a(ci, cj), tri_b(ci, cj)], 1)
    # Oblique rays toward the same vertices.
    d = rng.normal(size=(n, 3))
    d[:, 1] = -np.abs(d[:, 1]) - 0.5
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    org = v.astype(np.float64) - 15.0 * d
    obl = np.concatenate([org, np.zeros((n, 1)), d, np.full((n, 1), 3.4028234663852886e38)], 1).astype(np.float32)
    dev = ref.RefDevice(s, seed=0)
    out = {}
    for name, rays, inc in (("vertex", vert, incident_v), ("diagonal", diag, incident_d), ("oblique", obl, incident_v)):
        g, p, t, u, w = dev.trace(rays)
        ties = int(np.sum((g == 0) & np.any(p[:, None] == inc, 1)))
        out.update({f"{name}_rays": rays, f"{name}_geom": g, f"{name}_prim": p, f"{name}_t": t, f"{name}_u": u,
                    f"{name}_v": w, f"{name}_incident": inc.astype(np.int32), f"{name}_ties": np.int32(ties)})
        print(f"{name}: {ties} of {n} rays hit a triangle incident to the feature they aim at")
    dev.close()
    np.savez_compressed(OUT / "terrain_ties.npz", **out)


if __name__ == "__main__":
    which = sys.argv[1:] or ["terrain_rays", "cornell", "terrain"]
    if "terrain_rays" in which:
        make_terrain_rays()
    if "terrain_ties" in which:
        make_terrain_ties()
    if "cornell" in which:
        make_cornell()
    if "terrain" in which:
        make_terrain()
