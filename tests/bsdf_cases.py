"""Seeded BSDF parity tuples and the Standard-material cases they are evaluated on.

Shared by the BSDF parity tests and the fixture generator: tuples are (wo, wi, 3D sample) in
the canonical shading frame (N = z); wo is drawn mostly from the upper hemisphere (the side the
renderer shades from) with some grazing and below-horizon directions, wi from the full sphere.
"""
import numpy as np

import prt_types as T

GOLD_R = (1.0, 0.766, 0.336)
GOLD_G = (1.0, 0.95, 0.75)


def cases():
    """(name, material, medium id) for every lobe combination the device implements."""
    return [
        ("lambert", T.material(base_color=(0.7, 0.4, 0.2), specular_weight=0.0), 0),
        ("plastic_rough", T.material(base_color=(0.5, 0.6, 0.7), specular_roughness=0.3), 0),
        ("plastic_smooth", T.material(base_color=(0.5, 0.6, 0.7), specular_roughness=0.0), 0),
        ("gold_rough", T.material(metalness=1.0, base_color=GOLD_R, specular_color=GOLD_G, specular_roughness=0.25), 0),
        ("gold_smooth", T.material(metalness=1.0, base_color=GOLD_R, specular_color=GOLD_G, specular_roughness=0.0), 0),
        ("half_metal", T.material(metalness=0.5, base_color=(0.9, 0.5, 0.3), specular_roughness=0.4), 0),
        ("glass_rough_out", T.material(transmission_weight=1.0, specular_roughness=0.2), 0),
        ("glass_rough_in", T.material(transmission_weight=1.0, specular_roughness=0.2), 1),
        ("glass_smooth", T.material(transmission_weight=1.0, specular_roughness=0.0), 0),
        ("coat_rough_lambert", T.material(base_color=(0.3, 0.6, 0.3), specular_weight=0.0, coat_weight=1.0,
                                          coat_roughness=0.2), 0),
        ("coat_smooth_lambert", T.material(base_color=(0.3, 0.6, 0.3), specular_weight=0.0, coat_weight=1.0,
                                           coat_roughness=0.0), 0),
        ("coat_tinted_plastic", T.material(base_color=(0.8, 0.2, 0.2), coat_weight=0.7, coat_roughness=0.35,
                                           coat_color=(0.9, 0.8, 0.6)), 0),
        ("rough_diffuse", T.material(base_color=(0.6, 0.5, 0.4), specular_weight=0.0, diffuse_roughness=0.7), 0),
        ("rough_diffuse_plastic", T.material(base_color=(0.2, 0.5, 0.7), diffuse_roughness=0.4,
                                             specular_roughness=0.25), 0),
        ("sheen_lambert", T.material(base_color=(0.4, 0.3, 0.6), specular_weight=0.0, sheen_weight=0.8,
                                     sheen_color=(1.0, 0.9, 0.8), sheen_roughness=0.4), 0),
        ("sheen_coat_plastic", T.material(base_color=(0.7, 0.6, 0.2), specular_roughness=0.3, coat_weight=0.6,
                                          coat_roughness=0.2, sheen_weight=0.5, sheen_roughness=0.2), 0),
        ("sheen_gold", T.material(metalness=1.0, base_color=GOLD_R, specular_color=GOLD_G, specular_roughness=0.3,
                                  sheen_weight=1.0, sheen_roughness=0.6), 0),
        ("principled_plastic", T.principled(base_color=(0.6, 0.3, 0.2), specular_ior=1.5, specular_roughness=0.35), 0),
        ("principled_smooth_plastic", T.principled(base_color=(0.2, 0.4, 0.6), specular_ior=1.45, base_weight=0.8), 0),
        ("principled_metal", T.principled(base_color=GOLD_R, specular_color=GOLD_G, metalness=1.0,
                                          specular_roughness=0.3, base_weight=0.5), 0),
        ("principled_glass", T.principled(transmission_weight=1.0, specular_ior=1.5, specular_roughness=0.2), 0),
        ("principled_coat_sheen", T.principled(base_color=(0.3, 0.6, 0.4), specular_ior=1.5, specular_roughness=0.4,
                                               coat_weight=0.8, coat_roughness=0.1, coat_thickness=2.0,
                                               coat_color=(0.9, 0.7, 0.5), sheen_weight=0.7, sheen_tint=0.5,
                                               sheen_roughness=0.3), 0),
        ("subsurface_half", T.material(base_color=(0.6, 0.5, 0.4), specular_weight=0.0, subsurface_weight=0.5,
                                       subsurface_color=(0.9, 0.4, 0.3), subsurface_anisotropy=0.2), 0),
        ("subsurface_full_plastic", T.material(base_color=(0.6, 0.5, 0.4), specular_roughness=0.3,
                                               subsurface_weight=1.0, subsurface_color=(0.3, 0.8, 0.5),
                                               subsurface_anisotropy=-0.3), 0),
        ("subsurface_btdf_only", T.material(base_color=(0.5, 0.5, 0.5), specular_weight=0.0, subsurface_weight=0.7,
                                            subsurface_color=(0.8, 0.7, 0.2), subsurface_anisotropy=1.0), 0),
        ("subsurface_rough", T.material(base_color=(0.4, 0.6, 0.7), diffuse_roughness=0.5, specular_roughness=0.2,
                                        subsurface_weight=0.4, subsurface_color=(0.9, 0.9, 0.6)), 0),
        ("thin_glass_smooth", T.material(transmission_weight=1.0, thin_walled=1, specular_roughness=0.0,
                                         transmission_color=(0.8, 0.9, 0.7)), 0),
        ("thin_glass_rough", T.material(transmission_weight=1.0, thin_walled=1, specular_roughness=0.25,
                                        transmission_color=(0.7, 0.8, 0.9), transmission_depth=0.5), 0),
        ("thin_glass_coat", T.material(transmission_weight=0.8, thin_walled=1, specular_roughness=0.15,
                                       base_color=(0.6, 0.3, 0.3), coat_weight=0.5, coat_roughness=0.1), 0),
        ("transparent_ior1", T.material(transmission_weight=1.0, specular_ior=1.0), 0),
        ("half_transparent_ior1", T.material(transmission_weight=0.5, specular_ior=1.0, base_color=(0.2, 0.7, 0.4)), 0),
        ("opacity_lambert", T.material(base_color=(0.7, 0.5, 0.3), specular_weight=0.0, opacity=0.4), 0),
        ("opacity_coat_plastic", T.material(base_color=(0.3, 0.4, 0.8), specular_roughness=0.3, coat_weight=0.5,
                                            coat_roughness=0.2, opacity=0.7), 0),
        ("opacity_zero", T.material(base_color=(0.5, 0.5, 0.5), opacity=0.0), 0),
        ("principled_thin_backlight", T.principled(base_color=(0.7, 0.5, 0.3), specular_ior=1.5,
                                                   specular_roughness=0.3, thin_walled=1, backlight=0.8), 0),
        ("principled_thin_glass", T.principled(transmission_weight=1.0, specular_ior=1.5, specular_roughness=0.15,
                                               thin_walled=1, thickness=0.5, transmission_color=(0.9, 0.8, 0.6)), 0),
        ("principled_opacity", T.principled(base_color=(0.2, 0.6, 0.8), specular_ior=1.5, specular_roughness=0.3,
                                            opacity=0.6), 0),
    ]


def tuples(n, seed):
    rng = np.random.default_rng(seed)
    wo = rng.normal(size=(n, 3))
    wo /= np.linalg.norm(wo, axis=1, keepdims=True)
    flip = rng.uniform(size=n) < 0.9
    wo[flip, 2] = np.abs(wo[flip, 2])
    wi = rng.normal(size=(n, 3))
    wi /= np.linalg.norm(wi, axis=1, keepdims=True)
    s = rng.uniform(size=(n, 3))
    return np.concatenate([wo, wi, s], 1).astype(np.float32)


def compare(gpu, ref, rel=1e-5, floor=1e-6):
    """Per-tuple agreement of the 13 outputs.

    eval value and pdf, sample weight and pdf: |a - b| <= rel * max(|a|, |b|) + floor;
    sampled direction (a unit vector): |a - b| <= max(rel, 2e-5) per component; sample type:
    equal; and both sides must agree on whether sampling succeeded. Sample outputs are
    compared only where both succeeded. Returns boolean arrays {"eval", "sample", "flags"}."""
    def close(a, b):
        return np.abs(a - b) <= rel * np.maximum(np.abs(a), np.abs(b)) + floor

    out = {}
    out["eval"] = close(gpu[:, 0:4], ref[:, 0:4]).all(1)
    gs = np.max(gpu[:, 4:7], 1) > 0
    rs = np.max(ref[:, 4:7], 1) > 0
    both = gs & rs
    w_ok = close(gpu[:, 4:7], ref[:, 4:7]).all(1) & close(gpu[:, 10], ref[:, 10])
    wi_ok = (np.abs(gpu[:, 7:10] - ref[:, 7:10]) <= max(rel, 2e-5)).all(1)
    type_ok = gpu[:, 11].view(np.int32) == ref[:, 11].view(np.int32)
    out["sample"] = (gs == rs) & (~both | (w_ok & wi_ok & type_ok))
    out["flags"] = gpu[:, 12].view(np.int32) == ref[:, 12].view(np.int32)
    return out
