"""The voxel tool SDF built from a closed mesh (mpm_tool_sdf_build), restating
ToolSDF::build / buildFromVerts / computeSDFCPU (src/ToolSDF.cu:212-280,
:348-377, :379-532).  The reference's source does not compile with this
toolchain (a goto past initialisations in its closest-point routine), so its
builder cannot be run: the oracle restates it, including the reference's
interior case of the closest-point routine (a + u (b - a) + v (c - a),
u = 1 - v - w, where the published algorithm has a + v (b - a) + w (c - a)).

- CPU: the oracle against a numpy restatement written here (float32
  arithmetic in the same order) on a small box mesh: equal bit for bit;
- GPU: mpm_tool_sdf_build (distances and signs on the GPU, the in-place
  passes on the host) against the oracle on a 192-triangle cylinder: equal
  bit for bit, and the descriptor.
"""
from __future__ import annotations

import numpy as np
import pytest

f32 = np.float32
FMAX = np.finfo(np.float32).max


def box_mesh(h=(2e-4, 1.5e-4, 1e-4)):
    hx, hy, hz = h
    v = np.array([[sx * hx, sy * hy, sz * hz] for sz in (-1, 1) for sy in (-1, 1) for sx in (-1, 1)], np.float32)
    quads = [(0, 2, 3, 1), (4, 5, 7, 6), (0, 1, 5, 4), (2, 6, 7, 3), (0, 4, 6, 2), (1, 3, 7, 5)]
    t = np.array([[q[0], q[1], q[2]] for q in quads] + [[q[0], q[2], q[3]] for q in quads], np.int32)
    return v, t, outward_normals(v, t)


def cylinder_mesh(R=3e-4, L=4e-4, n=48):
    th = np.arange(n) * 2 * np.pi / n
    r0 = np.stack([R * np.cos(th), np.full(n, -L / 2), R * np.sin(th)], 1)
    r1 = np.stack([R * np.cos(th), np.full(n, L / 2), R * np.sin(th)], 1)
    v = np.concatenate([r0, r1, [[0, -L / 2, 0], [0, L / 2, 0]]]).astype(np.float32)
    c0, c1 = 2 * n, 2 * n + 1
    tris = []
    for i in range(n):
        j = (i + 1) % n
        tris += [[i, j, n + i], [j, n + j, n + i], [c0, j, i], [c1, n + i, n + j]]
    t = np.array(tris, np.int32)
    return v, t, outward_normals(v, t)


def outward_normals(v, t):
    a, b, c = (v[t[:, k]].astype(np.float64) for k in range(3))
    nr = np.cross(b - a, c - a)
    nr /= np.linalg.norm(nr, axis=1, keepdims=True)
    nr[((a + b + c) / 3 * nr).sum(1) < 0] *= -1
    return nr.astype(np.float32)


def closest_dist2(p, a, b, c):
    """Squared distance and closest point, float32, the reference's region tests."""
    dot = lambda u, w: f32(f32(f32(u[0] * w[0]) + f32(u[1] * w[1])) + f32(u[2] * w[2]))
    ab, ac, ap = b - a, c - a, p - a
    d1, d2 = dot(ab, ap), dot(ac, ap)
    if d1 <= 0 and d2 <= 0:
        q = a
    else:
        bp = p - b
        d3, d4 = dot(ab, bp), dot(ac, bp)
        vc = f32(f32(d1 * d4) - f32(d3 * d2))
        if d3 >= 0 and d4 <= d3:
            q = b
        elif vc <= 0 and d1 >= 0 and d3 <= 0:
            q = a + f32(d1 / f32(d1 - d3)) * ab
        else:
            cp = p - c
            d5, d6 = dot(ab, cp), dot(ac, cp)
            vb = f32(f32(d5 * d2) - f32(d1 * d6))
            va = f32(f32(d3 * d6) - f32(d5 * d4))
            if d6 >= 0 and d5 <= d6:
                q = c
            elif vb <= 0 and d2 >= 0 and d6 <= 0:
                q = a + f32(d2 / f32(d2 - d6)) * ac
            elif va <= 0 and f32(d4 - d3) >= 0 and f32(d5 - d6) >= 0:
                w = f32(f32(d4 - d3) / f32(f32(d4 - d3) + f32(d5 - d6)))
                q = b + w * (c - b)
            else:
                den = f32(f32(1) / f32(f32(va + vb) + vc))
                vv, ww = f32(vb * den), f32(vc * den)
                u = f32(f32(f32(1) - vv) - ww)
                q = (a + u * (b - a)) + vv * (c - a)
    d = p - q
    return dot(d, d), q


def build_numpy(v, t, nrm, padding, vpa):
    bmin, bmax = v.min(0) - f32(padding), v.max(0) + f32(padding)
    ext = bmax - bmin
    vox = f32(ext.max() / f32(vpa))
    dims = np.minimum((ext / vox).astype(np.int64) + 2, 256)
    nx, ny, nz = (int(d) for d in dims)
    g = np.full((nz, ny, nx), FMAX, np.float32)
    inv = f32(f32(1) / vox)
    centre = lambda ix, iy, iz: (bmin + (np.array([ix, iy, iz], np.float32) + f32(0.5)) * vox).astype(np.float32)
    for tri in t:
        a, b, c = v[tri[0]], v[tri[1]], v[tri[2]]
        lo, hi = np.minimum(np.minimum(a, b), c), np.maximum(np.maximum(a, b), c)
        i0 = np.maximum(0, ((lo - bmin) * inv).astype(np.int64) - 1)
        i1 = np.minimum(dims - 1, ((hi - bmin) * inv).astype(np.int64) + 2)
        for iz in range(i0[2], i1[2] + 1):
            for iy in range(i0[1], i1[1] + 1):
                for ix in range(i0[0], i1[0] + 1):
                    d2, _ = closest_dist2(centre(ix, iy, iz), a, b, c)
                    g[iz, iy, ix] = min(g[iz, iy, ix], d2)
    g = np.where(g < FMAX, np.sqrt(g), g).astype(np.float32)
    band = f32(vox * f32(2))
    for iz, iy, ix in np.argwhere(g <= band):
        p = centre(ix, iy, iz)
        best, bn, bq = FMAX, None, None
        for k, tri in enumerate(t):
            a, b, c = v[tri[0]], v[tri[1]], v[tri[2]]
            lo, hi = np.minimum(np.minimum(a, b), c), np.maximum(np.maximum(a, b), c)
            if (p < lo - vox).any() or (p > hi + vox).any():
                continue
            d2, q = closest_dist2(p, a, b, c)
            if d2 < best:
                best, bn, bq = d2, nrm[k], q
        if best < FMAX:
            d = p - bq
            if f32(f32(f32(d[0] * bn[0]) + f32(d[1] * bn[1])) + f32(d[2] * bn[2])) < 0:
                g[iz, iy, ix] = -g[iz, iy, ix]
    for _ in range(3):
        for iz in range(1, nz - 1):
            for iy in range(1, ny - 1):
                for ix in range(1, nx - 1):
                    if g[iz, iy, ix] < FMAX:
                        continue
                    nd = np.abs(g[iz - 1:iz + 2, iy - 1:iy + 2, ix - 1:ix + 2]).copy()
                    nd[1, 1, 1] = FMAX
                    m = nd.min()
                    if m < FMAX:
                        g[iz, iy, ix] = f32(m + f32(vox * f32(0.5)))
    g[g >= FMAX] = f32(vox * f32(max(nx, ny, nz)))
    return {"v": g, "origin": tuple(bmin), "voxel": float(vox)}


def test_oracle_build_matches_numpy_restatement(oracle):
    v, t, n = box_mesh()
    ref = build_numpy(v, t, n, 5e-5, 10)
    got = oracle.tool_sdf_build(v, t, n, 5e-5, 10)
    assert got["v"].shape == ref["v"].shape
    assert np.array_equal(np.float32(got["origin"]), np.float32(ref["origin"])) and got["voxel"] == ref["voxel"]
    assert np.array_equal(got["v"], ref["v"])
    # the field has both signs and values from every stage
    assert (got["v"] < 0).any() and (got["v"] > 0).any()


@pytest.mark.gpu
@pytest.mark.parametrize("mesh", ["box", "cylinder"])
def test_gpu_build_matches_oracle(oracle, mesh):
    from mpm_b200 import tool_sdf_build
    v, t, n = box_mesh() if mesh == "box" else cylinder_mesh()
    ours = tool_sdf_build(v, t, n, padding=1e-4, voxels_per_axis=40)
    ref = oracle.tool_sdf_build(v, t, n, 1e-4, 40)
    assert ours["v"].shape == ref["v"].shape
    assert np.array_equal(np.float32(ours["origin"]), np.float32(ref["origin"])) and ours["voxel"] == ref["voxel"]
    assert np.array_equal(ours["v"], ref["v"])
