"""Seeded synthetic scenes and ray sets for the five workloads.

Every generator is a pure function of its seed (numpy PCG64), so the CUDA path,
the CPU oracle and the reference build see byte-identical inputs.  No dataset
is named by the reference; these stand in for its scenes with the shapes and
value distributions of the workloads:

* ``displaced_octasphere`` -- triangle sphere: an octahedron subdivided k times
  (8 * 4**k faces; k = 7 gives 131,072), projected to the unit sphere and
  displaced radially by seeded value noise (amplitude 0.1).  ``nfaces``
  truncates the face list (used by the batched workload).
* ``tet_grid`` -- 64^3 cells in [0,1]^3, interior vertices jittered by
  U(+-0.2 cell), five tetrahedra per cell in alternating orientation
  (1,310,720 tets), plus a per-vertex scalar (sum of four Gaussians).
* ``particles`` -- centres U[0,1)^3, radii log-normal (median 1e-3,
  sigma 0.5), advected by a seeded smooth velocity field.
* ``volume_blobs`` -- a density grid as a sum of anisotropic Gaussian blobs,
  clamped to [0,1], plus an RGBA transfer-function table.
"""
from __future__ import annotations

import numpy as np

RAY_DTYPE = np.dtype([("org", "<f4", 3), ("prev_prim", "<u4"), ("dir", "<f4", 3),
                      ("prev_t", "<f4")])
MISS = 0xFFFFFFFF


# ---------------------------------------------------------------- triangles
def _value_noise(p, rng, lattice=8):
    """Trilinear value noise on a random lattice over [-1.5,1.5]^3, in [-1,1]."""
    g = rng.uniform(-1.0, 1.0, size=(lattice + 1,) * 3)
    q = (np.clip(p, -1.5, 1.5) + 1.5) / 3.0 * lattice
    i = np.minimum(np.floor(q).astype(np.int64), lattice - 1)
    f = q - i
    out = np.zeros(p.shape[0])
    for dz in (0, 1):
        for dy in (0, 1):
            for dx in (0, 1):
                w = ((f[:, 0] if dx else 1 - f[:, 0]) * (f[:, 1] if dy else 1 - f[:, 1])
                     * (f[:, 2] if dz else 1 - f[:, 2]))
                out += w * g[i[:, 0] + dx, i[:, 1] + dy, i[:, 2] + dz]
    return out


def octasphere(levels):
    """Unit octasphere: (vertices float64 (V,3), faces uint32 (F,3)); the
    children of face f are faces 4f..4f+3."""
    v = np.array([[1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1]],
                 np.float64)
    f = np.array([[0, 2, 4], [2, 1, 4], [1, 3, 4], [3, 0, 4],
                  [2, 0, 5], [1, 2, 5], [3, 1, 5], [0, 3, 5]], np.int64)
    for _ in range(levels):
        e = np.stack([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]], 1).reshape(-1, 2)
        key = np.minimum(e[:, 0], e[:, 1]) * (v.shape[0] + 1) + np.maximum(e[:, 0], e[:, 1])
        uk, inv = np.unique(key, return_inverse=True)
        a = uk // (v.shape[0] + 1)
        b = uk % (v.shape[0] + 1)
        mid = 0.5 * (v[a] + v[b])
        mid /= np.linalg.norm(mid, axis=1, keepdims=True)
        m = (inv.reshape(-1, 3) + v.shape[0])
        v = np.concatenate([v, mid])
        a0, a1, a2 = f[:, 0], f[:, 1], f[:, 2]
        m01, m12, m20 = m[:, 0], m[:, 1], m[:, 2]
        f = np.stack([np.stack([a0, m01, m20], 1), np.stack([m01, a1, m12], 1),
                      np.stack([m20, m12, a2], 1), np.stack([m01, m12, m20], 1)],
                     1).reshape(-1, 3)
    return v, f.astype(np.uint32)


def displaced_octasphere(levels=7, seed=123456, amplitude=0.1, nfaces=None):
    """(vertices float32 (V,3), faces uint32 (F,3))."""
    rng = np.random.default_rng(seed)
    v, f = octasphere(levels)
    r = 1.0 + amplitude * _value_noise(v, rng)
    verts = (v * r[:, None]).astype(np.float32)
    if nfaces is not None:
        f = f[:nfaces]
    return verts, np.ascontiguousarray(f)


def octasphere_for_count(n, seed):
    """Truncated displaced octasphere with exactly n faces."""
    levels = 0
    while 8 * 4 ** levels < n:
        levels += 1
    return displaced_octasphere(levels, seed=seed, nfaces=n)


# ---------------------------------------------------------------- tetrahedra
# corner c = x + 2y + 4z of a cube cell; five tets per cell in two parities
_TETS_EVEN = [(0, 1, 2, 4), (3, 2, 1, 7), (5, 4, 7, 1), (6, 7, 4, 2), (1, 2, 4, 7)]
_TETS_ODD = [(1, 0, 5, 3), (2, 3, 6, 0), (4, 5, 0, 6), (7, 6, 3, 5), (0, 3, 5, 6)]


def tet_grid(cells=64, seed=123456, jitter=0.2, orient=-1):
    """(vertices float32 (V,3), tets uint32 (N,4), scalar float32 (V,)).

    Every tetrahedron is ordered so that det(v1-v0, v2-v0, v3-v0) has the sign
    ``orient``; -1 is the orientation for which the reference's Pluecker test
    (render/render_accel_tetra.cc:243-567) reports the entering face first."""
    rng = np.random.default_rng(seed)
    n1 = cells + 1
    g = np.stack(np.meshgrid(np.arange(n1), np.arange(n1), np.arange(n1),
                             indexing="ij"), -1).reshape(-1, 3)  # (x,y,z), x slowest
    h = 1.0 / cells
    p = g * h
    interior = np.all((g > 0) & (g < cells), axis=1)
    p[interior] += rng.uniform(-jitter * h, jitter * h, size=(interior.sum(), 3))
    verts = p.astype(np.float32)

    def vid(x, y, z):
        return (x * n1 + y) * n1 + z

    cx, cy, cz = np.meshgrid(np.arange(cells), np.arange(cells), np.arange(cells),
                             indexing="ij")
    cx, cy, cz = cx.ravel(), cy.ravel(), cz.ravel()
    corner = np.stack([vid(cx + (c & 1), cy + ((c >> 1) & 1), cz + ((c >> 2) & 1))
                       for c in range(8)], 1)
    par = (cx + cy + cz) & 1
    te = corner[:, np.array(_TETS_EVEN)]  # (cells^3, 5, 4)
    to = corner[:, np.array(_TETS_ODD)]
    tets = np.where(par[:, None, None] == 0, te, to).reshape(-1, 4).astype(np.int64)
    v = verts.astype(np.float64)
    d = np.linalg.det(np.stack([v[tets[:, 1]] - v[tets[:, 0]], v[tets[:, 2]] - v[tets[:, 0]],
                                v[tets[:, 3]] - v[tets[:, 0]]], 1))
    flip = np.sign(d) != orient
    tets[flip, 1], tets[flip, 2] = tets[flip, 2].copy(), tets[flip, 1].copy()
    # scalar field: sum of four seeded isotropic Gaussians
    cen = rng.uniform(0.2, 0.8, size=(4, 3))
    wid = rng.uniform(0.1, 0.3, size=4)
    amp = rng.uniform(0.5, 1.0, size=4)
    s = np.zeros(v.shape[0])
    for k in range(4):
        s += amp[k] * np.exp(-np.sum((v - cen[k]) ** 2, 1) / (2 * wid[k] ** 2))
    return verts, tets.astype(np.uint32), s.astype(np.float32)


# ---------------------------------------------------------------- particles
def particles(n=16_777_216, seed=123456, median_radius=1e-3, sigma=0.5):
    """(centres float32 (n,3), radii float32 (n,))."""
    rng = np.random.default_rng(seed)
    pos = rng.random((n, 3), dtype=np.float32)
    rad = (median_radius * np.exp(sigma * rng.standard_normal(n))).astype(np.float32)
    return pos, rad


class VelocityField:
    """Seeded smooth velocity field: a few random Fourier modes."""

    def __init__(self, seed=7, modes=4, speed=2e-3):
        rng = np.random.default_rng(seed)
        self.k = rng.normal(0, 2.0 * np.pi, size=(modes, 3)).astype(np.float32)
        self.ph = rng.uniform(0, 2 * np.pi, size=(modes, 3)).astype(np.float32)
        self.a = (speed * rng.normal(size=(modes, 3)) / np.sqrt(modes)).astype(np.float32)

    def advect(self, pos, dt=1.0):
        v = np.zeros_like(pos)
        for m in range(self.k.shape[0]):
            arg = pos @ self.k[m]
            for c in range(3):
                v[:, c] += self.a[m, c] * np.sin(arg + self.ph[m, c])
        return (pos + dt * v).astype(np.float32)

    def advect_torch(self, pos, dt=1.0):
        """The same step on a torch tensor (device-side frame generation)."""
        import torch
        k = torch.as_tensor(self.k, device=pos.device)
        v = torch.zeros_like(pos)
        for m in range(self.k.shape[0]):
            arg = pos @ k[m]
            for c in range(3):
                v[:, c] += float(self.a[m, c]) * torch.sin(arg + float(self.ph[m, c]))
        return pos + dt * v


def particle_frames(pos, nframes=10, seed=7, device=None):
    """Centres of `nframes` frames: frame 0 = pos, frame f+1 = frame f advected
    by VelocityField(seed); torch tensors on `device`."""
    import torch
    vf = VelocityField(seed)
    frames = [torch.as_tensor(pos, device=device)]
    for _ in range(nframes - 1):
        frames.append(vf.advect_torch(frames[-1]).contiguous())
    return frames


# ---------------------------------------------------------------- rays
def _normalize(d):
    return d / np.linalg.norm(d, axis=-1, keepdims=True)


def pinhole_rays(width, height, eye, lookat, up=(0, 1, 0), fov_deg=45.0):
    """One ray per pixel centre, row-major from the top row; pinhole camera
    with vertical field of view fov_deg (the frame of render/render_camera.cc:17-63)."""
    eye = np.asarray(eye, np.float64)
    look = np.asarray(lookat, np.float64) - eye
    u = _normalize(np.cross(look, up))
    v = _normalize(np.cross(look, u))
    look = _normalize(look)
    flen = 0.5 * height / np.tan(0.5 * np.radians(fov_deg))
    corner = flen * look + eye - 0.5 * (width * u + height * v)
    px = np.arange(width) + 0.5
    py = np.arange(height) + 0.5
    P = corner[None, None] + px[None, :, None] * u + py[:, None, None] * v
    d = _normalize(P - eye).astype(np.float32).reshape(-1, 3)
    rays = np.zeros(width * height, RAY_DTYPE)
    rays["org"] = eye.astype(np.float32)
    rays["dir"] = d
    rays["prev_prim"] = MISS
    return rays


def make_rays(org, dirs):
    """Ray records from (n, 3) origins and directions (not normalised)."""
    rays = np.zeros(len(org), RAY_DTYPE)
    rays["org"] = np.asarray(org, np.float32)
    rays["dir"] = np.asarray(dirs, np.float32)
    rays["prev_prim"] = MISS
    return rays


def ortho_rays(width, height, lo=(0.0, 0.0), hi=(1.0, 1.0), z=2.0):
    """Orthographic rays along -z through pixel centres of [lo,hi]^2."""
    xs = lo[0] + (np.arange(width) + 0.5) * (hi[0] - lo[0]) / width
    ys = lo[1] + (np.arange(height) + 0.5) * (hi[1] - lo[1]) / height
    X, Y = np.meshgrid(xs, ys)
    rays = np.zeros(width * height, RAY_DTYPE)
    rays["org"][:, 0] = X.ravel()
    rays["org"][:, 1] = Y.ravel()
    rays["org"][:, 2] = z
    rays["dir"][:, 2] = -1.0
    rays["prev_prim"] = MISS
    return rays


def hemisphere_dirs(normals, seed):
    """Uniform directions on the hemisphere about each normal."""
    rng = np.random.default_rng(seed)
    n = normals.shape[0]
    d = rng.normal(size=(n, 3))
    d = _normalize(d)
    s = np.sign(np.sum(d * normals, 1))
    s[s == 0] = 1.0
    return (d * s[:, None]).astype(np.float32)


# ---------------------------------------------------------------- volume
def volume_blobs(res=256, nblobs=32, seed=123456, shift_voxels=0.0):
    """Density grid (res,res,res) float32 (z slowest, x fastest) in [0,1]:
    the blob sum scaled down, when it exceeds 0.95, to peak at 0.95 -- no
    plateau of texels on the transfer function's upper clamp, where the
    density gradient has a kink (one-sided derivatives differ)."""
    rng = np.random.default_rng(seed)
    cen = rng.uniform(0.2, 0.8, size=(nblobs, 3))
    cen = cen + shift_voxels / (res - 1)
    sig = rng.uniform(0.03, 0.12, size=(nblobs, 3))
    amp = rng.uniform(0.3, 0.9, size=nblobs)
    x = np.linspace(0.0, 1.0, res)
    out = np.zeros((res, res, res), np.float32)
    for b in range(nblobs):
        gx = np.exp(-0.5 * ((x - cen[b, 0]) / sig[b, 0]) ** 2)
        gy = np.exp(-0.5 * ((x - cen[b, 1]) / sig[b, 1]) ** 2)
        gz = np.exp(-0.5 * ((x - cen[b, 2]) / sig[b, 2]) ** 2)
        out += (amp[b] * gz[:, None, None] * gy[None, :, None] * gx[None, None, :]).astype(np.float32)
    peak = float(out.max())
    if peak > 0.95:
        out *= np.float32(0.95 / peak)
    return out.astype(np.float32)


def transfer_function(entries=256, seed=123456):
    """RGBA table (entries, 4) float32: smooth colour ramp, opacity rising
    with density."""
    rng = np.random.default_rng(seed)
    x = np.linspace(0.0, 1.0, entries)
    ph = rng.uniform(0, 2 * np.pi, size=3)
    rgb = 0.5 + 0.5 * np.sin(2 * np.pi * x[:, None] * np.array([1.0, 1.3, 1.7]) + ph)
    a = np.clip((x - 0.05) * 1.2, 0.0, 1.0) ** 1.5
    return np.concatenate([rgb, a[:, None]], 1).astype(np.float32)


# ---------------------------------------------------------------- batched
_OCTA_CACHE: dict = {}


def _octa(levels):
    if levels not in _OCTA_CACHE:
        _OCTA_CACHE[levels] = octasphere(levels)
    return _OCTA_CACHE[levels]


def batched_scenes(nscenes=64, seed=2024, lo=1e3, hi=1e6, sizes=(128, 256, 512, 1024),
                   min_faces=1024):
    """Uneven triangle scenes for the batched build+trace.

    Scene s: a displaced octasphere truncated to n_s faces, n_s log-uniform in
    [lo, hi] (at least ``min_faces``, the size from which Build32 applies),
    seen by a square pinhole image of a side drawn uniformly from ``sizes``
    (camera at distance 3 on +z, 45 degree field of view).  Returns a dict with
    the concatenated ``vertices``, ``faces`` (vertex ids into the concatenated
    vertices), ``rays``, the nscenes+1 ``face_offsets`` / ``ray_offsets``, and
    per-scene ``counts`` and ``sides``."""
    rng = np.random.default_rng(seed)
    counts = np.exp(rng.uniform(np.log(lo), np.log(hi), nscenes)).astype(np.int64)
    counts = np.maximum(counts, min_faces)
    sides = rng.choice(np.asarray(sizes), nscenes)
    verts, faces, rays = [], [], []
    fo, ro = [0], [0]
    vbase = 0
    for s in range(nscenes):
        n = int(counts[s])
        levels = 0
        while 8 * 4 ** levels < n:
            levels += 1
        v, f = _octa(levels)
        srng = np.random.default_rng([seed, s])
        r = 1.0 + 0.1 * _value_noise(v, srng)
        vs = (v * r[:, None]).astype(np.float32)
        fs = f[:n]
        verts.append(vs)
        faces.append(fs.astype(np.uint64) + vbase)
        vbase += vs.shape[0]
        fo.append(fo[-1] + n)
        side = int(sides[s])
        rays.append(pinhole_rays(side, side, (0, 0, 3), (0, 0, 0)))
        ro.append(ro[-1] + side * side)
    faces = np.concatenate(faces)
    assert faces.max() < 2 ** 32
    return dict(vertices=np.concatenate(verts), faces=faces.astype(np.uint32),
                rays=np.concatenate(rays), face_offsets=np.asarray(fo, np.uint64),
                ray_offsets=np.asarray(ro, np.uint64), counts=counts, sides=sides)


# ---------------------------------------------------------------- secondaries
def _mix64(z):
    z = (z ^ (z >> np.uint64(30))) * np.uint64(0xbf58476d1ce4e5b9)
    z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94d049bb133111eb)
    return z ^ (z >> np.uint64(31))


def spawn_secondary_np(rays, hits, normals, seed):
    """NumPy statement of srt_spawn_secondary (the particle workload's bounce):
    for every hit ray, in order, a ray from the hit point (float32
    org + t * dir) in a uniform hemisphere direction about the unit normal,
    with prev_prim / prev_t of the hit.  Directions are computed in float64
    here (the device computes in float32), so they agree to ~1e-6.
    Returns (rays RAY_DTYPE (k,), unit normals float32 (k, 3))."""
    hit = np.nonzero(hits["prim"] != MISS)[0]
    n = np.asarray(normals, np.float64)[hit]
    n /= np.linalg.norm(n, axis=1, keepdims=True)
    with np.errstate(over="ignore"):
        z = _mix64(np.uint64(seed) + np.uint64(0x9e3779b97f4a7c15) * (hit.astype(np.uint64)
                                                                     + np.uint64(1)))
    u1 = (z >> np.uint64(40)).astype(np.float64) / 16777216.0
    u2 = ((z >> np.uint64(16)) & np.uint64(0xffffff)).astype(np.float64) / 16777216.0
    ct = u1
    st = np.sqrt(np.maximum(0.0, 1.0 - ct * ct))
    lx, ly = st * np.cos(2 * np.pi * u2), st * np.sin(2 * np.pi * u2)
    sg = np.where(np.signbit(n[:, 2]), -1.0, 1.0)
    a = -1.0 / (sg + n[:, 2])
    b = n[:, 0] * n[:, 1] * a
    b1 = np.stack([1.0 + sg * n[:, 0] ** 2 * a, sg * b, -sg * n[:, 0]], 1)
    b2 = np.stack([b, sg + n[:, 1] ** 2 * a, -n[:, 1]], 1)
    d = lx[:, None] * b1 + ly[:, None] * b2 + ct[:, None] * n
    out = np.zeros(hit.size, RAY_DTYPE)
    out["org"] = rays["org"][hit] + hits["t"][hit, None] * rays["dir"][hit]
    out["dir"] = d.astype(np.float32)
    out["prev_prim"] = hits["prim"][hit]
    out["prev_t"] = hits["t"][hit]
    return out, n.astype(np.float32)


def sphere_normals_np(rays, hits, centers):
    """Unit normals at sphere hits (zero for misses): normalize(p - centre)
    with p = org + t * dir in float32."""
    nrm = np.zeros((rays.size, 3), np.float32)
    hit = np.nonzero(hits["prim"] != MISS)[0]
    p = rays["org"][hit] + hits["t"][hit, None] * rays["dir"][hit]
    v = (p - centers[hits["prim"][hit]]).astype(np.float64)
    nrm[hit] = (v / np.linalg.norm(v, axis=1, keepdims=True)).astype(np.float32)
    return nrm


# ---------------------------------------------------------------- scenes
def affine(rotation_axis=(0.0, 0.0, 1.0), angle_deg=0.0, scale=(1.0, 1.0, 1.0),
           translate=(0.0, 0.0, 0.0)):
    """4x4 in Matrixd's layout (p' = (p, 1) m; translation in the last row)
    for p' = R diag(scale) p + translate, R the rotation about the axis."""
    a = np.asarray(rotation_axis, np.float64)
    a = a / np.linalg.norm(a)
    th = np.radians(angle_deg)
    K = np.array([[0, -a[2], a[1]], [a[2], 0, -a[0]], [-a[1], a[0], 0]])
    R = np.eye(3) + np.sin(th) * K + (1 - np.cos(th)) * (K @ K)
    A = R @ np.diag(np.asarray(scale, np.float64))
    m = np.eye(4)
    m[:3, :3] = A.T
    m[3, :3] = translate
    return m


def scene_elements(seed=31, ntri=3, nsph=2, ntet=1, spread=4.0, nline=0, nsolid=0):
    """A mixed scene: ntri displaced octaspheres, nsph particle clouds, ntet
    tetrahedral grids, nline hair-strand line sets and nsolid solid grids
    (hexahedra, prisms, pyramids in turn), each under a seeded rotation,
    (non-uniform) scale and translation inside [-spread, spread]^3.  Returns
    a list of dicts with kind (0 tri, 1 tet, 2 sphere, 3 lines, 4 solids),
    verts, faces (tri, tet), radius (sphere, lines), segments (lines), nv
    (solids) and T."""
    rng = np.random.default_rng(seed)
    out = []
    kinds = [0] * ntri + [2] * nsph + [1] * ntet + [3] * nline + [4] * nsolid
    for j, k in enumerate(kinds):
        T = affine(rng.normal(size=3), rng.uniform(0, 360),
                   rng.uniform(0.5, 1.5, size=3), rng.uniform(-spread, spread, size=3))
        if k == 0:
            v, f = displaced_octasphere(3 + j % 2, seed=seed + j)
            out.append(dict(kind=0, verts=v, faces=f, T=T))
        elif k == 2:
            p, r = particles(2000 + 500 * j, seed=seed + j, median_radius=0.02)
            out.append(dict(kind=2, verts=p, radius=r, T=T))
        elif k == 3:
            p, sg, r = line_strands(150 + 50 * (j % 3), 8, seed=seed + j, radius=0.03)
            out.append(dict(kind=3, verts=p, segments=sg, radius=r, T=T))
        elif k == 4:  # 1024 solids or more: the reference's Build32 range
            nv = (8, 6, 5)[j % 3]
            v, ix = solid_grid(nv, {8: 11, 6: 8, 5: 6}[nv], seed=seed + j)
            out.append(dict(kind=4, verts=v - np.float32(0.5), faces=ix, nv=nv, T=T))
        else:
            v, f, _ = tet_grid(4 + j % 3, seed=seed + j)
            out.append(dict(kind=1, verts=v, faces=f, T=T))
    return out


def scene_rays(n, bmin, bmax, seed=5, boxes=None):
    """Rays from a sphere around the box to seeded points inside it, or
    inside one of ``boxes`` ((lo, hi) arrays of shape (m, 3)) picked per ray,
    with a share of axis-aligned directions."""
    rng = np.random.default_rng(seed)
    bmin = np.asarray(bmin, np.float64)
    bmax = np.asarray(bmax, np.float64)
    c = 0.5 * (bmin + bmax)
    rad = 0.75 * np.linalg.norm(bmax - bmin)
    o = c + rad * _normalize(rng.normal(size=(n, 3)))
    if boxes is None:
        tgt = bmin + rng.uniform(size=(n, 3)) * (bmax - bmin)
    else:
        lo, hi = (np.asarray(b, np.float64) for b in boxes)
        k = rng.integers(0, lo.shape[0], size=n)
        tgt = lo[k] + (0.25 + 0.5 * rng.uniform(size=(n, 3))) * (hi[k] - lo[k])
    d = _normalize(tgt - o)
    ax = rng.uniform(size=n) < 0.1  # axis-aligned: zero direction components
    if ax.any():
        k = rng.integers(0, 3, size=ax.sum())
        dd = np.zeros((ax.sum(), 3))
        dd[np.arange(ax.sum()), k] = np.where(rng.uniform(size=ax.sum()) < 0.5, -1.0, 1.0)
        d[ax] = dd
        o[ax] = tgt[ax] - rad * dd
    rays = np.zeros(n, RAY_DTYPE)
    rays["org"] = o.astype(np.float32)
    rays["dir"] = d.astype(np.float32)
    rays["prev_prim"] = MISS
    return rays


def instanced_scene(seed=77, grid=4, spacing=3.0):
    """grid^3 elements on a lattice of the given spacing, each an instance of
    one of three accels (131,072-triangle octasphere, 1,000,000-sphere cloud,
    32^3-cell tetrahedral grid), centred, scaled to about 2 units, rotated
    and jittered.  Returns dict(accels=[{kind, verts, faces|radius}],
    elements=[{accel, T}], prims=[per-element primitive count])."""
    rng = np.random.default_rng(seed)
    v, f = displaced_octasphere(7)
    p, r = particles(1_000_000, seed=seed, median_radius=0.004)
    tv, tf, _ = tet_grid(32, seed=seed)
    accels = [dict(kind=0, verts=v, faces=f, centre=(0.0, 0.0, 0.0), size=2.2),
              dict(kind=2, verts=p, radius=r, centre=(0.5, 0.5, 0.5), size=1.0),
              dict(kind=1, verts=tv, faces=tf, centre=(0.5, 0.5, 0.5), size=1.0)]
    nprim = [f.shape[0], p.shape[0], tf.shape[0]]
    elements, prims = [], []
    off = 0.5 * (grid - 1) * spacing
    for j in range(grid ** 3):
        a = j % 3
        cell = np.array(np.unravel_index(j, (grid,) * 3), np.float64) * spacing - off
        s = 2.0 / accels[a]["size"] * rng.uniform(0.8, 1.2)
        C = np.eye(4)
        C[3, :3] = -np.asarray(accels[a]["centre"])
        M = affine(rng.normal(size=3), rng.uniform(0, 360), (s, s, s),
                   cell + rng.uniform(-0.3, 0.3, size=3))
        elements.append(dict(accel=a, T=C @ M))
        prims.append(nprim[a])
    return dict(accels=accels, elements=elements, prims=prims)


# ---------------------------------------------------------------- textures
def dense_texture(fmt, dims=(9, 7, 5), comps=1, seed=1):
    """A seeded 3D texture (D, H, W, comps) of format 0 byte, 1 float, 2 double."""
    rng = np.random.default_rng(seed)
    w, h, d = dims
    shape = (d, h, w, comps) if comps > 1 else (d, h, w)
    if fmt == 0:
        return rng.integers(0, 256, size=shape, dtype=np.uint8)
    x = rng.random(shape)
    return x.astype(np.float32 if fmt == 1 else np.float64)


def remap_table(n, seed=2, power=1.7):
    """A monotone coordinate remap of n entries in [0, 1] (stretched toward
    one end, as non-uniform grids are)."""
    rng = np.random.default_rng(seed)
    t = np.sort(rng.random(n)) ** power
    t[0], t[-1] = 0.0, 1.0
    return t.astype(np.float32)


def sparse_blocks(fmt, comps, nblocks=12, seed=3, gdim=(64, 48, 40), overlap=False):
    """Seeded sparse volume: blocks at random integer offsets (non-overlapping
    on a lattice, or overlapping), extents 4-16 and voxel sizes that differ
    from the extents.  Returns (blocks BLOCK-layout structured array, pool bytes,
    gdim)."""
    rng = np.random.default_rng(seed)
    dt = np.dtype([("offset", "<i4", 3), ("extent", "<i4", 3), ("size", "<i4", 3),
                   ("level", "<i4"), ("data_offset", "<u8")])
    b = np.zeros(nblocks, dt)
    itemsize = {0: 1, 1: 4, 2: 8}[fmt]
    chunks, off = [], 0
    cells = [(i, j, k) for i in range(4) for j in range(3) for k in range(2)]
    rng.shuffle(cells)
    for n in range(nblocks):
        ext = rng.integers(4, 17, size=3)
        if overlap:
            o = rng.integers(0, np.array(gdim) - ext)
        else:
            c = np.array(cells[n % len(cells)])
            o = c * np.array([16, 16, 20])
        size = rng.integers(2, 9, size=3)
        b[n]["offset"], b[n]["extent"], b[n]["size"] = o, ext, size
        b[n]["data_offset"] = off
        nvox = int(np.prod(size)) * min(comps, 4)
        if fmt == 0:
            data = rng.integers(0, 256, size=nvox, dtype=np.uint8)
        else:
            data = rng.random(nvox).astype(np.float32 if fmt == 1 else np.float64)
        raw = data.tobytes()
        raw += b"\0" * ((-len(raw)) % 16)
        chunks.append(raw)
        off += len(raw)
    return b, b"".join(chunks), tuple(int(x) for x in gdim)


def exp_coord_map(n):
    """A non-uniform coordinate map of n entries: exp(4 i / n) normalised to
    [0, 1] (the stretched axis of the reference's non-uniform volume example)."""
    m = np.exp(4.0 * (np.arange(n, dtype=np.float32) / np.float32(n))).astype(np.float32)
    return ((m - m[0]) / (m[-1] - m[0])).astype(np.float32)


def sparse_pages(ndiv=16, page=32, seed=123456):
    """A sparse volume of committed pages in a 3D checkerboard (the layout of
    the reference's sparse_volume_render example, which commits the pages
    with (x + y + z) even out of 2x2x2): ndiv^3 page slots of page^3 byte
    texels, half of them committed, each with its own seeded smooth-ish
    content.  Returns (blocks, pool bytes, global dims)."""
    rng = np.random.default_rng(seed)
    dt = np.dtype([("offset", "<i4", 3), ("extent", "<i4", 3), ("size", "<i4", 3),
                   ("level", "<i4"), ("data_offset", "<u8")])
    slots = [(x, y, z) for z in range(ndiv) for y in range(ndiv) for x in range(ndiv)
             if (x + y + z) % 2 == 0]
    b = np.zeros(len(slots), dt)
    nv = page ** 3
    g = np.arange(page, dtype=np.float32) / page
    base = (np.sin(6.0 * g)[None, None, :] + np.cos(5.0 * g)[None, :, None]
            + np.sin(4.0 * g + 1.0)[:, None, None])
    pool = np.empty(len(slots) * nv, np.uint8)
    for n, (x, y, z) in enumerate(slots):
        b[n]["offset"] = (x * page, y * page, z * page)
        b[n]["extent"] = (page, page, page)
        b[n]["size"] = (page, page, page)
        b[n]["data_offset"] = n * nv
        a, c = rng.random(2).astype(np.float32)
        pool[n * nv:(n + 1) * nv] = np.clip(40.0 * (base * (0.5 + a) + 3.0 * c), 0,
                                            255).astype(np.uint8).reshape(-1)
    return b, pool.tobytes(), (ndiv * page,) * 3


def march_coords(w=512, h=512, steps=64):
    """Texture coordinates of a shader march: w x h parallel rays tilted by
    (0.2, 0.1) per unit depth, `steps` samples each from r = 1 down to 0,
    ray-major ((ray, step) -> ray * steps + step), all inside [0, 1)^3.
    Returns (w * h * steps, 3) float32."""
    x = (0.8 * (np.arange(w, dtype=np.float32) + 0.5) / w).astype(np.float32)
    y = (0.9 * (np.arange(h, dtype=np.float32) + 0.5) / h).astype(np.float32)
    s = ((np.arange(steps, dtype=np.float32) + 0.5) / steps).astype(np.float32)
    out = np.empty((h, w, steps, 3), np.float32)
    out[..., 0] = x[None, :, None] + np.float32(0.2) * s[None, None, :]
    out[..., 1] = y[:, None, None] + np.float32(0.1) * s[None, None, :]
    out[..., 2] = np.float32(1.0) - s[None, None, :]
    return out.reshape(-1, 3)


def sparse_table(offsets, extents, sizes, fmt, comps, seed):
    """A block table (BLOCK layout) and data pool from per-block offsets,
    extents and voxel sizes, with seeded texels."""
    rng = np.random.default_rng(seed)
    dt = np.dtype([("offset", "<i4", 3), ("extent", "<i4", 3), ("size", "<i4", 3),
                   ("level", "<i4"), ("data_offset", "<u8")])
    b = np.zeros(len(offsets), dt)
    chunks, off = [], 0
    for i, (o, e, z) in enumerate(zip(offsets, extents, sizes)):
        b[i]["offset"], b[i]["extent"], b[i]["size"] = o, e, z
        b[i]["data_offset"] = off
        nv = int(np.prod(z)) * min(comps, 4)
        data = (rng.integers(0, 256, size=nv, dtype=np.uint8) if fmt == 0 else
                rng.random(nv).astype(np.float32 if fmt == 1 else np.float64))
        raw = data.tobytes()
        raw += b"\0" * ((-len(raw)) % 16)
        chunks.append(raw)
        off += len(raw)
    return b, b"".join(chunks)


LOCATE_CASES = ("crowded", "negative", "single", "nested", "slabs", "unit")


def sparse_locate_case(case, fmt, comps):
    """Block layouts that stress BVHTree::Locate: crowded (80 overlapping
    blocks in 40^3, more than 16 reaching into many cells), negative offsets,
    a single block, nested blocks (one around all), long thin slabs.
    Returns (blocks, pool, global dims)."""
    rng = np.random.default_rng({"crowded": 1, "negative": 2, "single": 3, "nested": 4,
                                 "slabs": 5, "unit": 6}[case])
    if case == "crowded":
        n = 80
        ext = rng.integers(3, 17, size=(n, 3))
        off = rng.integers(0, 40 - ext)
        gdim = (40, 40, 40)
    elif case == "negative":
        n = 30
        ext = rng.integers(4, 12, size=(n, 3))
        off = rng.integers(-37, 20, size=(n, 3))
        gdim = (33, 29, 41)
    elif case == "single":
        n = 1
        ext = np.array([[7, 5, 9]])
        off = np.array([[3, -2, 1]])
        gdim = (16, 16, 16)
    elif case == "nested":
        n = 25
        ext = rng.integers(2, 10, size=(n, 3))
        off = rng.integers(1, 30, size=(n, 3))
        ext[0], off[0] = (40, 40, 40), (0, 0, 0)
        ext[5], off[5] = (20, 20, 20), (10, 10, 10)
        gdim = (40, 40, 40)
    elif case == "slabs":
        n = 24
        ext = np.where(rng.random((n, 3)) < 0.3, rng.integers(50, 200, size=(n, 3)),
                       rng.integers(1, 4, size=(n, 3)))
        off = rng.integers(0, 60, size=(n, 3))
        gdim = (128, 128, 128)
    else:  # one voxel per unit (size == extent) around the origin, both signs
        n = 27
        ext = rng.integers(2, 9, size=(n, 3))
        off = rng.integers(-12, 8, size=(n, 3))
        off[0], ext[0] = (-4, -4, -4), (8, 8, 8)
        gdim = (24, 24, 24)
    sizes = rng.integers(1, 9, size=(n, 3))
    if case == "unit":
        sizes = ext.copy()
        sizes[1::3] = rng.integers(1, 9, size=sizes[1::3].shape)
    blocks, pool = sparse_table(off, ext, sizes, fmt, comps, seed=n + fmt)
    return blocks, pool, gdim


def sparse_edge_coords(blocks, gdim, n, seed, spread=(0.0, 1.0)):
    """Coordinates on block faces, edges and corners, a few float ulps and
    the block tree's 1e-6 widening off them, inside blocks, and (n / 4 more)
    uniform in `spread`.  (n + n // 4, 3) float32."""
    rng = np.random.default_rng(seed)
    g = np.array(gdim, np.float64)
    b = blocks[rng.integers(0, blocks.size, size=n)]
    corner = b["offset"] + b["extent"] * rng.integers(0, 2, size=(n, 3))
    inner = b["offset"] + rng.random((n, 3)) * b["extent"]
    pos = np.where(rng.integers(0, 2, size=(n, 3)).astype(bool), corner, inner)
    nudge = np.array([0, 0, 1e-6, -1e-6, 2e-6, -2e-6, 1e-7])[rng.integers(0, 7, size=(n, 3))]
    u = ((pos + nudge * b["extent"]) / g).astype(np.float32)
    ulps = rng.integers(-2, 3, size=(n, 3))
    for k in (-2, -1, 1, 2):
        to = np.float32(np.inf if k > 0 else -np.inf)
        step = np.nextafter(u, to).astype(np.float32)
        if abs(k) == 2:
            step = np.nextafter(step, to).astype(np.float32)
        u = np.where(ulps == k, step, u)
    anywhere = rng.uniform(*spread, size=(n // 4, 3)).astype(np.float32)
    # tiny coordinates of both signs around the origin
    tiny = np.array([0.0, -0.0, 1e-30, -1e-30, 1e-12, -1e-12, 1e-7, -1e-7, 2e-38, -2e-38],
                    np.float32)
    special = tiny[rng.integers(0, tiny.size, size=(max(n // 16, 16), 3))]
    return np.concatenate([u, anywhere, special]).astype(np.float32)


def line_strands(nstrands=2000, nseg=16, seed=123456, radius=0.004, taper=True):
    """Seeded hair-like strands for the line (capped cylinder) accel:
    `nstrands` polylines of `nseg` segments rooted on the unit sphere,
    growing outward with a random bend.  Returns (positions (V, 3) float32,
    segments (nstrands * nseg, 2) uint32 vertex pairs, per-vertex radius
    (V,) float32)."""
    rng = np.random.default_rng(seed)
    root = rng.normal(size=(nstrands, 3))
    root /= np.linalg.norm(root, axis=1, keepdims=True)
    d = root + 0.3 * rng.normal(size=(nstrands, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    pts = np.empty((nstrands, nseg + 1, 3), np.float64)
    pts[:, 0] = root
    step = 0.6 / nseg
    for j in range(1, nseg + 1):
        d = d + 0.25 * rng.normal(size=(nstrands, 3))
        d /= np.linalg.norm(d, axis=1, keepdims=True)
        pts[:, j] = pts[:, j - 1] + step * d
    pos = pts.reshape(-1, 3).astype(np.float32)
    base = np.arange(nstrands)[:, None] * (nseg + 1) + np.arange(nseg)[None, :]
    seg = np.stack([base, base + 1], axis=-1).reshape(-1, 2).astype(np.uint32)
    w = (1.0 - 0.7 * np.arange(nseg + 1) / nseg) if taper else np.ones(nseg + 1)
    rad = (radius * np.tile(w, nstrands)).astype(np.float32)
    return pos, seg, rad


def line_segments(n=20000, seed=7, extent=1.0, radius=(0.002, 0.02)):
    """Seeded independent segments of random length and direction in a cube,
    radii per vertex (different at the two ends), with a few zero-length and
    coincident segments."""
    rng = np.random.default_rng(seed)
    a = rng.uniform(-extent, extent, size=(n, 3))
    b = a + rng.normal(scale=0.08 * extent, size=(n, 3))
    b[: n // 50] = a[: n // 50]  # zero length
    a[n // 50: n // 25] = a[n // 25: n // 25 + (n // 25 - n // 50)]  # shared start points
    pos = np.stack([a, b], axis=1).reshape(-1, 3).astype(np.float32)
    seg = np.arange(2 * n, dtype=np.uint32).reshape(n, 2)
    rad = rng.uniform(*radius, size=2 * n).astype(np.float32)
    return pos, seg, rad


def line_cases():
    """Small line sets with the shapes that stress LineAccel: (name, positions,
    segments, radius or None, constant radius, options dict, rays)."""
    out = []
    rng = np.random.default_rng(11)
    # axis-aligned segments, rays along the axes (zero direction components),
    # rays along a segment's own axis (through both caps), rays from inside
    pos = np.array([[0, 0, 0], [1, 0, 0], [0, 0.5, 0], [0, 0.5, 1], [0.5, -0.5, 0.5],
                    [0.5, 1.5, 0.5], [2, 2, 2], [2, 2, 2]], np.float32)
    seg = np.array([[0, 1], [2, 3], [4, 5], [6, 7]], np.uint32)
    rad = np.array([0.1, 0.2, 0.15, 0.15, 0.05, 0.3, 0.2, 0.2], np.float32)
    o = []
    for x in np.linspace(-0.5, 2.5, 13):
        for y in np.linspace(-0.7, 2.3, 13):
            o.append(((x, y, -3.0), (0.0, 0.0, 1.0)))
            o.append(((-3.0, y, x), (1.0, 0.0, 0.0)))
            o.append(((x, -3.0, y), (0.0, 1.0, 0.0)))
    o += [((-2.0, 0.0, 0.0), (1.0, 0.0, 0.0)), ((3.0, 0.0, 0.0), (-1.0, 0.0, 0.0)),
          ((0.0, 0.5, -2.0), (0.0, 0.0, 1.0)), ((0.5, 0.0, 0.0), (0.0, 0.3, 1.0)),
          ((0.5, 0.02, 0.01), (1.0, 0.0, 0.0)), ((0.5, 0.5, 0.5), (0.0, 1.0, 0.0)),
          ((2.0, 2.0, 0.0), (0.0, 0.0, 1.0)), ((2.0, 2.0, 2.0), (0.0, 0.0, -1.0))]
    rays = make_rays(np.array([a for a, _ in o], np.float32), np.array([b for _, b in o], np.float32))
    for cap in (True, False):
        out.append((f"axes-cap{int(cap)}", pos, seg, rad, 0.0, dict(cap=cap), rays))
    # one, two and three lines (the root is a leaf), constant radius
    for n in (1, 2, 3):
        out.append((f"tiny{n}", pos[:2 * n], np.arange(2 * n, dtype=np.uint32).reshape(n, 2),
                    None, 0.12, {}, rays))
    # a chain of lines at midpoints 2^-k: every spatial split peels one off
    k = np.arange(90, dtype=np.float64)
    a = np.stack([2.0 ** -k, np.zeros_like(k), np.zeros_like(k)], 1)
    b = a + np.array([0.0, 0.0, 2.0 ** -20])
    pos2 = np.stack([a, b], 1).reshape(-1, 3).astype(np.float32)
    seg2 = np.arange(2 * k.size, dtype=np.uint32).reshape(-1, 2)
    eye = rng.uniform(-0.5, 1.5, size=(2000, 3)).astype(np.float32)
    tgt = np.stack([2.0 ** -rng.uniform(0, 40, 2000), np.zeros(2000), np.zeros(2000)], 1)
    rays2 = make_rays(eye, (tgt - eye).astype(np.float32))
    out.append(("chain", pos2, seg2, None, 2.0 ** -22, dict(min_leaf=1), rays2))
    # random segments with leaf and depth limits
    p3, s3, r3 = line_segments(3000, seed=5)
    eye = rng.uniform(-2, 2, size=(4000, 3)).astype(np.float32)
    d = rng.normal(size=(4000, 3)).astype(np.float32)
    rays3 = make_rays(eye, d)
    out.append(("limits", p3, s3, r3, 0.0, dict(min_leaf=7, max_depth=6), rays3))
    out.append(("leaf1", p3, s3, r3, 0.0, dict(min_leaf=1), rays3))
    return out


# hexahedron corner order: 0..3 the bottom face, 4..7 above them
_HEX_CORNERS = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0],
                         [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]])
# pyramid bases from the hexahedron's faces (base b0..b3, apex at the cell centre)
_PYR_BASES = [(0, 1, 2, 3), (4, 7, 6, 5), (0, 4, 5, 1), (1, 5, 6, 2), (2, 6, 7, 3), (0, 3, 7, 4)]


def solid_grid(nv, g, seed=3, jitter=0.2):
    """Seeded solids filling the unit cube: g^3 cells of a jittered grid as
    hexahedra (nv = 8), two prisms per cell (nv = 6) or six pyramids around
    the cell centre (nv = 5).  Returns (vertices (V, 3) float32, indices
    (N, nv) uint32)."""
    rng = np.random.default_rng(seed)
    ax = np.arange(g + 1, dtype=np.float64) / g
    X, Y, Z = np.meshgrid(ax, ax, ax, indexing="ij")
    P = np.stack([X, Y, Z], -1)
    inner = np.zeros(P.shape[:3], bool)
    inner[1:-1, 1:-1, 1:-1] = True
    P[inner] += rng.uniform(-jitter, jitter, size=(inner.sum(), 3)) / g
    verts = P.reshape(-1, 3)
    c = np.stack(np.meshgrid(np.arange(g), np.arange(g), np.arange(g), indexing="ij"), -1)
    c = c.reshape(-1, 3)
    corner = c[:, None, :] + _HEX_CORNERS[None]
    hexa = (corner[..., 0] * (g + 1) + corner[..., 1]) * (g + 1) + corner[..., 2]
    if nv == 8:
        return verts.astype(np.float32), hexa.astype(np.uint32)
    if nv == 6:
        a = hexa[:, [0, 1, 2, 4, 5, 6]]
        b = hexa[:, [0, 2, 3, 4, 6, 7]]
        return verts.astype(np.float32), np.concatenate([a, b]).astype(np.uint32)
    centre = verts[hexa].mean(axis=1)
    cid = verts.shape[0] + np.arange(hexa.shape[0])
    pyr = [np.concatenate([hexa[:, list(b)], cid[:, None]], 1) for b in _PYR_BASES]
    return (np.concatenate([verts, centre]).astype(np.float32),
            np.concatenate(pyr).astype(np.uint32))


def solid_rays(n_side=96, seed=5):
    """Rays for the solid tests: grid-aligned orthographic rays through
    vertex planes (ties at shared faces and edges), pinhole rays, and rays
    starting inside the cube in random directions."""
    o1 = ortho_rays(n_side, n_side, (-0.05, -0.05), (1.05, 1.05), z=1.5)
    xs = (np.arange(n_side // 2) + 0.5) / (n_side // 2)
    X, Y = np.meshgrid(xs, xs)
    o2 = make_rays(np.stack([X.ravel(), np.full(X.size, -0.5), Y.ravel()], 1),
                   np.tile([0.0, 1.0, 0.0], (X.size, 1)))
    p = pinhole_rays(n_side, n_side, (1.7, 1.3, 2.1), (0.5, 0.5, 0.5), fov_deg=50)
    rng = np.random.default_rng(seed)
    org = rng.uniform(0.05, 0.95, size=(n_side * n_side // 2, 3))
    d = rng.normal(size=org.shape)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    inside = make_rays(org, d)
    return np.concatenate([o1, o2, p, inside])
