"""Test scenes built through the public scene API (this project's own
scenes; the reference's testscenes module is not available)."""
from __future__ import annotations

import numpy as np

SLOT_BASE, SLOT_MR, SLOT_NORMAL, SLOT_EMISSIVE = 0, 1, 2, 3


def quad_tris(a, b, c, d):
    return np.array([a, b, c, a, c, d], dtype=np.float32).reshape(2, 9)


def sphere(radius: float, n_lon: int, n_lat: int, center=(0.0, 0.0, 0.0)):
    """UV sphere as a triangle soup with normals and uv0 (outward)."""
    pos, nrm, uv = [], [], []
    cx, cy, cz = center

    def v(i, j):
        th = np.pi * j / n_lat
        ph = 2.0 * np.pi * i / n_lon
        n = np.array([np.sin(th) * np.cos(ph), np.cos(th), np.sin(th) * np.sin(ph)])
        return n * radius + np.array([cx, cy, cz]), n, (i / n_lon, j / n_lat)

    for j in range(n_lat):
        for i in range(n_lon):
            a, b, c, d = v(i, j), v(i + 1, j), v(i + 1, j + 1), v(i, j + 1)
            for tri in ((a, b, c), (a, c, d)):
                for p, n, t in tri:
                    pos.append(p)
                    nrm.append(n)
                    uv.append(t)
    pos = np.array(pos, np.float32).reshape(-1, 3, 3)
    nrm = np.array(nrm, np.float32).reshape(-1, 3, 3)
    uv = np.array(uv, np.float32).reshape(-1, 3, 2)
    # Wind every triangle outwards (front faces out) and drop the
    # degenerate pole triangles.
    cr = np.cross(pos[:, 1] - pos[:, 0], pos[:, 2] - pos[:, 0])
    out = np.einsum("ij,ij->i", cr, pos.mean(axis=1) - np.array(center, np.float32))
    flip = out < 0
    for arr in (pos, nrm, uv):
        arr[flip, 1], arr[flip, 2] = arr[flip, 2].copy(), arr[flip, 1].copy()
    keep = np.linalg.norm(cr, axis=1) > 1e-9
    return pos[keep].reshape(-1, 9), nrm[keep].reshape(-1, 9), uv[keep].reshape(-1, 6)


def checker(size=64, cells=8, alpha=None):
    y, x = np.mgrid[0:size, 0:size]
    t = ((x * cells // size + y * cells // size) & 1).astype(np.float32)
    rgba = np.zeros((size, size, 4), np.float32)
    rgba[..., 0] = 0.9 * t + 0.1
    rgba[..., 1] = 0.6 * t + 0.2
    rgba[..., 2] = 0.3 + 0.5 * (1 - t)
    rgba[..., 3] = 1.0 if alpha is None else alpha(x, y, t)
    return rgba


def add_floor_and_light(pkg, s, light=(6.0, 5.5, 5.0), floor_mat=None):
    fm = s.add_material(floor_mat or pkg.material(base_color=(0.7, 0.7, 0.7, 1), metallic=0.0, roughness=0.8))
    s.add_mesh(quad_tris((-3, 0, 3), (3, 0, 3), (3, 0, -3), (-3, 0, -3)), fm)
    lm = s.add_material(pkg.material(base_color=(0, 0, 0, 1), metallic=0.0, emissive=light, has_specular=1,
                                     specular=0.0))
    s.add_mesh(quad_tris((-0.8, 2.5, -0.8), (0.8, 2.5, -0.8), (0.8, 2.5, 0.8), (-0.8, 2.5, 0.8)), lm)


def materials_scene(pkg):
    """Floor, emissive quad, point light and five spheres exercising the
    layered BSDF: volume glass, thin transmission, clearcoat, sheen, metal."""
    s = pkg.Scene()
    add_floor_and_light(pkg, s)
    mats = [
        pkg.material(base_color=(0.95, 0.95, 1.0, 1), metallic=0.0, roughness=0.1, has_transmission=1,
                     transmission=1.0, has_volume=1, thickness=1.0, attenuation_distance=1.5,
                     attenuation_color=(0.6, 0.8, 0.9)),
        pkg.material(base_color=(0.9, 0.7, 0.5, 1), metallic=0.0, roughness=0.3, has_transmission=1,
                     transmission=0.8),
        pkg.material(base_color=(0.6, 0.1, 0.1, 1), metallic=0.0, roughness=0.6, has_clearcoat=1, clearcoat=1.0,
                     clearcoat_roughness=0.15),
        pkg.material(base_color=(0.1, 0.1, 0.3, 1), metallic=0.0, roughness=0.9, has_sheen=1,
                     sheen_color=(0.9, 0.8, 0.6), sheen_roughness=0.5),
        pkg.material(base_color=(0.95, 0.8, 0.5, 1), metallic=1.0, roughness=0.35),
    ]
    for i, m in enumerate(mats):
        mid = s.add_material(m)
        pos, nrm, uv = sphere(0.45, 24, 12, center=(-1.6 + 0.8 * i, 0.45, 0.0))
        s.add_mesh(pos, mid, normals=nrm, uv0=uv)
    s.add_light(1, position=(2.0, 2.0, 2.0), color=(1.0, 0.9, 0.8), intensity=6.0)
    s.add_camera((0.0, 1.6, 4.2), (0.0, 0.4, 0.0), 0.8)
    return s


def textured_scene(pkg, min_filter=5, wrap=(2, 2), mag_linear=True, tex_size=256):
    """Checker-textured floor seen at a grazing angle (ray-cone LOD,
    trilinear filtering) plus a textured, tangent-mapped sphere. A small
    `tex_size` makes texels larger than pixels near the camera, so camera
    hits there take the magnification filter (LOD <= 0)."""
    s = pkg.Scene()
    t0 = s.add_texture(checker(tex_size, max(2, tex_size // 16)), srgb_encoded=True, wrap=wrap,
                       mag_linear=mag_linear, min_filter=min_filter)
    nm = np.zeros((64, 64, 4), np.float32)
    yy, xx = np.mgrid[0:64, 0:64]
    nm[..., 0] = 0.5 + 0.3 * np.sin(xx / 4.0)
    nm[..., 1] = 0.5 + 0.3 * np.cos(yy / 5.0)
    nm[..., 2] = 1.0
    nm[..., 3] = 1.0
    t1 = s.add_texture(nm, wrap=(1, 0), min_filter=3)
    m = pkg.material(base_color=(1, 1, 1, 1), metallic=0.0, roughness=0.7, tex={SLOT_BASE: (t0, 0)})
    m.tex[SLOT_BASE].transform[0] = 6.0
    m.tex[SLOT_BASE].transform[4] = 6.0
    fm = s.add_material(m)
    floor = quad_tris((-4, 0, 4), (4, 0, 4), (4, 0, -4), (-4, 0, -4))
    uv = np.array([[0, 1, 1, 1, 1, 0], [0, 1, 1, 0, 0, 0]], np.float32)
    s.add_mesh(floor, fm, uv0=uv)
    sm = s.add_material(pkg.material(base_color=(0.8, 0.8, 0.8, 1), metallic=0.0, roughness=0.4,
                                     tex={SLOT_BASE: (t0, 0), SLOT_NORMAL: (t1, 0)}))
    pos, nrm, uvs = sphere(0.6, 24, 12, center=(0.0, 0.6, 0.0))
    tan = np.zeros((pos.shape[0], 12), np.float32)
    tan.reshape(-1, 3, 4)[..., 0] = 1.0
    tan.reshape(-1, 3, 4)[..., 3] = 1.0
    s.add_mesh(pos, sm, normals=nrm, tangents=tan, uv0=uvs)
    s.add_light(0, direction=(-0.3, -1.0, -0.4), intensity=2.5)
    s.add_camera((0.0, 0.9, 4.0), (0.0, 0.3, 0.0), 0.9)
    return s


def alpha_scene(pkg):
    """Two MASK and one BLEND plane (texture alpha) over a floor, lit by an
    area light: exercises any-hit acceptance and BLEND coins."""
    s = pkg.Scene()
    add_floor_and_light(pkg, s)
    tex = s.add_texture(checker(64, 8, alpha=lambda x, y, t: 0.15 + 0.8 * t), wrap=(2, 2), min_filter=1)
    for i, (mode, cut) in enumerate(((1, 0.5), (2, 0.0), (1, 0.3))):
        m = pkg.material(base_color=(0.9, 0.5 + 0.2 * i, 0.3, 0.8), metallic=0.0, roughness=0.6, alpha_mode=mode,
                         alpha_cutoff=cut, double_sided=int(i == 1), tex={SLOT_BASE: (tex, 0)})
        mid = s.add_material(m)
        x = -1.2 + 1.2 * i
        q = quad_tris((x - 0.5, 0.0, 0.3 * i), (x + 0.5, 0.0, 0.3 * i), (x + 0.5, 1.2, 0.3 * i),
                      (x - 0.5, 1.2, 0.3 * i))
        uv = np.array([[0, 1, 1, 1, 1, 0], [0, 1, 1, 0, 0, 0]], np.float32)
        s.add_mesh(q, mid, uv0=uv)
    s.add_camera((0.3, 1.2, 3.8), (0.0, 0.5, 0.0), 0.9)
    return s


def sky(w=64, h=32):
    """Equirectangular sky: blue gradient with a bright sun patch."""
    img = np.zeros((h, w, 4), np.float32)
    t = (np.arange(h, dtype=np.float32) / h)[:, None]
    img[..., 0] = 0.3 + 0.4 * t
    img[..., 1] = 0.5 + 0.3 * t
    img[..., 2] = 0.9
    img[..., 3] = 1.0
    img[6:8, 40:43, :3] = (80.0, 70.0, 55.0)
    return img


def env_scene(pkg):
    """Spheres on a floor under the sky map and no other light."""
    s = pkg.Scene()
    fm = s.add_material(pkg.material(base_color=(0.6, 0.6, 0.6, 1), metallic=0.0, roughness=0.9))
    s.add_mesh(quad_tris((-3, 0, 3), (3, 0, 3), (3, 0, -3), (-3, 0, -3)), fm)
    for i in range(3):
        mid = s.add_material(pkg.material(base_color=(0.3 + 0.3 * i, 0.5, 0.8 - 0.2 * i, 1), metallic=float(i == 2),
                                          roughness=0.2 + 0.3 * i))
        pos, nrm, uv = sphere(0.4, 16, 8, center=(-1.0 + i, 0.4, 0.0))
        s.add_mesh(pos, mid, normals=nrm, uv0=uv)
    s.add_camera((0.0, 1.2, 3.5), (0.0, 0.3, 0.0), 0.8)
    return s


def psnr_rgb8(a: np.ndarray, b: np.ndarray) -> float:
    """PSNR over the RGB bytes of two RGBA8 images."""
    d = a[..., :3].astype(np.float64) - b[..., :3].astype(np.float64)
    mse = float(np.mean(d * d))
    return float("inf") if mse == 0 else 10.0 * np.log10(255.0 * 255.0 / mse)
