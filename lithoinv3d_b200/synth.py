"""Seeded synthetic models, station grids and data for the benchmark and the
parity tests.

* `icosphere_model` -- one closed icosphere body, radially perturbed
  (the single-body case: subdivision 3 gives 642 vertices / 1280 triangles).
* `voxel_contact_model` -- lithology groups labelled on a voxel grid by
  thresholding a sum of seeded Gaussian blobs; closed group volumes are built
  from voxel faces between different labels and from the grid boundary, each
  quad split along its first diagonal, so neighbouring groups share vertex
  positions exactly (the voxel-face extraction of the reference's Python
  preprocessing, python/lithoseed/src/lithoseed/_surfaces.py:394-615,
  restated here with explicit outward orientation).
* `station_grid` -- regular station grids.

Nothing here is timed; the generators only shape the inputs.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

from .api import FIXED, Z_ONLY, XYZ_FREE, Context, Model

# --------------------------------------------------------------- geometry --


def icosphere(subdiv: int):
    """Unit icosphere with outward (counter-clockwise seen from outside) faces."""
    t = (1.0 + 5.0 ** 0.5) / 2.0
    v = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
         (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    verts = [np.array(p, float) / np.linalg.norm(p) for p in v]
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
             (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11),
             (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    for _ in range(subdiv):
        mid = {}

        def m(a, b):
            k = (min(a, b), max(a, b))
            if k not in mid:
                p = verts[a] + verts[b]
                verts.append(p / np.linalg.norm(p))
                mid[k] = len(verts) - 1
            return mid[k]

        nf = []
        for a, b, c in faces:
            ab, bc, ca = m(a, b), m(b, c), m(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = nf
    V = np.array(verts)
    F = np.array(faces, dtype=np.int32)
    if signed_volume(V, F) < 0:
        F = F[:, [0, 2, 1]].copy()
    return V, F


def signed_volume(V: np.ndarray, F: np.ndarray) -> float:
    a, b, c = V[F[:, 0]], V[F[:, 1]], V[F[:, 2]]
    return float(np.einsum("ij,ij->i", a, np.cross(b, c)).sum() / 6.0)


def station_grid(n: int, spacing: float, z: float, center=(0.0, 0.0), ny: Optional[int] = None) -> np.ndarray:
    ny = n if ny is None else ny
    xs = center[0] + (np.arange(n) - (n - 1) / 2.0) * spacing
    ys = center[1] + (np.arange(ny) - (ny - 1) / 2.0) * spacing
    X, Y = np.meshgrid(xs, ys, indexing="xy")
    return np.stack([X.ravel(), Y.ravel(), np.full(X.size, float(z))], axis=1)


def blob_labels(shape, n_groups: int, n_blobs: int, rng: np.random.Generator, width=(0.1, 0.3)) -> np.ndarray:
    """Labels 0..n_groups-1 from quantile thresholds of a sum of Gaussian blobs."""
    nx, ny, nz = shape
    gx, gy, gz = np.meshgrid((np.arange(nx) + 0.5) / nx, (np.arange(ny) + 0.5) / ny, (np.arange(nz) + 0.5) / nz,
                             indexing="ij")
    fieldv = np.zeros(shape)
    for _ in range(n_blobs):
        c = rng.uniform(0, 1, 3)
        s = rng.uniform(*width)
        a = rng.uniform(0.5, 1.5) * rng.choice([-1.0, 1.0])
        fieldv += a * np.exp(-((gx - c[0]) ** 2 + (gy - c[1]) ** 2 + (gz - c[2]) ** 2) / (2 * s * s))
    qs = np.quantile(fieldv, np.linspace(0, 1, n_groups + 1)[1:-1])
    return np.digitize(fieldv, qs).astype(np.int32)


def voxel_group_volumes(labels: np.ndarray, cell: float, origin=(0.0, 0.0, 0.0)):
    """Closed outward-oriented triangle meshes, one per label value.

    Vertex (i, j, k) of the lattice sits at (x0 + i*cell, y0 + j*cell,
    z0 - k*cell) (k counts downward from the top surface z0).  Returns a list
    of (vertices[n,3], triangles[m,3], lattice[n,3]) per label 0..max."""
    nx, ny, nz = labels.shape
    G = int(labels.max()) + 1
    quads = [[] for _ in range(G)]  # (corner lattice coords [4,3], outward axis vector)
    padded = np.full((nx + 2, ny + 2, nz + 2), -1, dtype=np.int32)
    padded[1:-1, 1:-1, 1:-1] = labels
    # axis 0: faces at lattice i between cells i-1 and i
    for axis in range(3):
        lo = [slice(0, -1) if a == axis else slice(1, -1) for a in range(3)]
        hi = [slice(1, None) if a == axis else slice(1, -1) for a in range(3)]
        la = padded[tuple(lo)]
        lb = padded[tuple(hi)]
        diff = np.argwhere(la != lb)
        for idx in diff:
            a_lab = la[tuple(idx)]
            b_lab = lb[tuple(idx)]
            base = idx.copy()  # lattice coordinate of the face (along axis: position idx[axis])
            u, w = [d for d in range(3) if d != axis]
            c0 = base.copy()
            c1 = base.copy(); c1[u] += 1
            c2 = base.copy(); c2[u] += 1; c2[w] += 1
            c3 = base.copy(); c3[w] += 1
            corners = np.array([c0, c1, c2, c3])
            # cell a is on the low side of the plane along `axis`: its outward normal is +axis (lattice)
            if a_lab >= 0:
                quads[a_lab].append((corners, axis, +1))
            if b_lab >= 0:
                quads[b_lab].append((corners, axis, -1))
    out = []
    for g in range(G):
        lat_list = []
        tri_list = []
        for corners, axis, sgn in quads[g]:
            world = _lattice_to_world(corners, cell, origin)
            n = np.cross(world[1] - world[0], world[2] - world[0])
            # desired outward normal in world coordinates (lattice k points down)
            want = np.zeros(3)
            want[axis] = sgn * (-1.0 if axis == 2 else 1.0)
            if np.dot(n, want) < 0:
                corners = corners[[0, 3, 2, 1]]
            lat_list.append(corners)
        if not lat_list:
            out.append((np.zeros((0, 3)), np.zeros((0, 3), np.int32), np.zeros((0, 3), np.int64)))
            continue
        lat = np.array(lat_list).reshape(-1, 3)
        uniq, inv = np.unique(lat, axis=0, return_inverse=True)
        inv = inv.reshape(-1, 4)
        tris = np.concatenate([inv[:, [0, 1, 2]], inv[:, [0, 2, 3]]], axis=1).reshape(-1, 3)
        V = _lattice_to_world(uniq, cell, origin)
        out.append((V, tris.astype(np.int32), uniq))
    return out


def _lattice_to_world(lat: np.ndarray, cell: float, origin) -> np.ndarray:
    lat = np.asarray(lat, dtype=np.float64)
    return np.stack([origin[0] + lat[..., 0] * cell, origin[1] + lat[..., 1] * cell, origin[2] - lat[..., 2] * cell],
                    axis=-1)


# ---------------------------------------------------------------- problems --


@dataclass
class Problem:
    name: str
    densities: List[float]
    susceptibilities: List[float]
    meshes: List[tuple]  # (V, F, freedom)
    grav_xyz: np.ndarray
    mag_xyz: Optional[np.ndarray]
    inducing: tuple = (60.0, 0.0, 55000.0)  # inclination deg, declination deg, nT
    axis_scale: float = 1.0
    cp_stride: int = 0
    depth_bounds: Optional[tuple] = None
    extra: dict = field(default_factory=dict)
    station_groups: Optional[List[int]] = None  # batched bodies: stations per group, in group order

    def build_model(self) -> Model:
        m = Model()
        for g, (rho, chi) in enumerate(zip(self.densities, self.susceptibilities)):
            m.add_group(g, rho, chi)
        for g, (V, F, fr) in enumerate(self.meshes):
            m.set_group_mesh(g, V, F, fr)
        if self.axis_scale != 1.0:
            for ax in range(3):
                m.set_axis_scale(ax, self.axis_scale)
        if self.depth_bounds is not None:
            m.set_depth_bounds(*self.depth_bounds)
        if self.cp_stride > 0:
            m.set_control_point_stride(self.cp_stride)
        if len(self.meshes) > 1 and self.station_groups is None:
            m.build_shared_vertex_sync()
        return m

    def n_triangles(self) -> int:
        return int(sum(len(F) for _, F, _ in self.meshes))

    def make_context(self, model: Model, device: int = 0, grav_obs=None, grav_std=None, mag_obs=None,
                     mag_std=None) -> Context:
        ctx = Context(device)
        ctx.set_model(model)
        if self.station_groups is not None:
            ctx.set_station_groups(self.station_groups)
        ctx.set_field(*self.inducing)
        ctx.set_gravity_data(self.grav_xyz, grav_obs, grav_std)
        if self.mag_xyz is not None:
            ctx.set_magnetic_data(self.mag_xyz, mag_obs, mag_std)
        return ctx


def icosphere_model(subdiv=3, radius=200.0, center=(0.0, 0.0, -500.0), sigma=20.0, seed=1, n_side=40,
                    spacing=50.0, height=1.0, density=0.3, susceptibility=0.02, freedom=Z_ONLY,
                    axis_scale=1.0, joint=True) -> Problem:
    """Single closed icosphere body: radius 200 m centred at 500 m depth,
    vertices perturbed radially by N(0, sigma) from `seed`; n_side^2 stations
    at `spacing` metres, `height` above the flat surface z = 0."""
    rng = np.random.default_rng(seed)
    U, F = icosphere(subdiv)
    r = radius + rng.normal(0.0, sigma, len(U))
    V = np.asarray(center) + U * r[:, None]
    st = station_grid(n_side, spacing, height)
    return Problem("icosphere", [density], [susceptibility], [(V, F, freedom)], st, st if joint else None,
                   axis_scale=axis_scale)


def voxel_contact_model(shape=(24, 24, 12), cell=100.0, n_groups=4, n_blobs=6, seed=3, n_side=64, height=1.0,
                        cp_stride=4, freedom_interior=Z_ONLY, joint=True, axis_scale=1.0,
                        blob_width=(0.1, 0.3)) -> Problem:
    """Multi-unit contact model: groups labelled on a voxel grid by
    thresholding a sum of seeded Gaussian blobs; voxel-face closed volumes;
    densities U(-0.3, 0.5) g/cc, susceptibilities U(0, 0.05) SI; an
    n_side x n_side station grid over the footprint at `height`.  Vertices on
    the flat top (z = 0) and the base are fixed, every other vertex moves in z."""
    rng = np.random.default_rng(seed)
    labels = blob_labels(shape, n_groups, n_blobs, rng, width=blob_width)
    nx, ny, nz = shape
    origin = (-nx * cell / 2.0, -ny * cell / 2.0, 0.0)
    vols = voxel_group_volumes(labels, cell, origin)
    meshes = []
    for V, F, lat in vols:
        fr = np.full(len(V), freedom_interior, np.uint8)
        fr[(lat[:, 2] == 0) | (lat[:, 2] == nz)] = FIXED
        meshes.append((V, F, fr))
    rho = list(rng.uniform(-0.3, 0.5, n_groups))
    chi = list(rng.uniform(0.0, 0.05, n_groups))
    spacing = nx * cell / n_side
    st = station_grid(n_side, spacing, height, ny=int(round(ny * cell / spacing)))
    p = Problem("voxel", rho, chi, meshes, st, st if joint else None, cp_stride=cp_stride, axis_scale=axis_scale)
    p.extra["labels"] = labels
    return p


def topography(xy: np.ndarray, rng: np.random.Generator, n_waves: int = 8, amplitude: float = 80.0) -> np.ndarray:
    """Seeded sum of n_waves plane sinusoids, scaled into [0, amplitude] m."""
    z = np.zeros(len(xy))
    span = float(np.max(xy.max(0) - xy.min(0)))
    for _ in range(n_waves):
        k = rng.uniform(1.0, 6.0) * 2 * np.pi / span
        th = rng.uniform(0, 2 * np.pi)
        z += rng.uniform(0.3, 1.0) * np.sin(k * (xy[:, 0] * np.cos(th) + xy[:, 1] * np.sin(th)) + rng.uniform(0, 2 * np.pi))
    z -= z.min()
    return amplitude * z / max(z.max(), 1e-30)


def large_model(shape=(60, 60, 30), cell=100.0, n_groups=6, n_blobs=20, seed=5, n_side=200, cp_stride=4,
                blob_width=(0.05, 0.15)) -> Problem:
    """Large single inversion: the contact-model construction on a 60x60x30
    grid of 100 m voxels with 6 units (~194k triangles), x/y/z-free interior
    vertices, and an
    n_side^2 station grid whose heights follow a seeded topography (sum of 8
    sinusoids, 0-80 m above the flat top, plus 1 m)."""
    p = voxel_contact_model(shape=shape, cell=cell, n_groups=n_groups, n_blobs=n_blobs, seed=seed, n_side=n_side,
                            cp_stride=cp_stride, freedom_interior=XYZ_FREE, blob_width=blob_width)
    st = p.grav_xyz.copy()
    st[:, 2] = 1.0 + topography(st[:, :2], np.random.default_rng(seed + 100))
    p.grav_xyz = st
    p.mag_xyz = st
    p.name = "large"
    return p


# ------------------------------------------------------------ batched bodies --


def latlong_sphere(n_lat: int, n_lon: int):
    """Closed unit sphere: two poles and (n_lat - 1) rings of n_lon vertices;
    2 n_lon (n_lat - 1) triangles, outward."""
    V = [(0.0, 0.0, 1.0)]
    for i in range(1, n_lat):
        th = np.pi * i / n_lat
        for j in range(n_lon):
            ph = 2 * np.pi * j / n_lon
            V.append((np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), np.cos(th)))
    V.append((0.0, 0.0, -1.0))
    V = np.array(V)
    south = len(V) - 1

    def ring(i, j):
        return 1 + (i - 1) * n_lon + (j % n_lon)

    F = []
    for j in range(n_lon):
        F.append((0, ring(1, j), ring(1, j + 1)))
    for i in range(1, n_lat - 1):
        for j in range(n_lon):
            a, b, c, d = ring(i, j), ring(i, j + 1), ring(i + 1, j), ring(i + 1, j + 1)
            F.append((a, c, d))
            F.append((a, d, b))
    for j in range(n_lon):
        F.append((south, ring(n_lat - 1, j + 1), ring(n_lat - 1, j)))
    F = np.array(F, dtype=np.int32)
    if signed_volume(V, F) < 0:
        F = F[:, [0, 2, 1]].copy()
    return V, F


def star_prism(n_poly: int, n_layers: int, rng: np.random.Generator):
    """Closed prism over a random star-shaped polygon (radius 0.6-1.0 at
    n_poly sorted angles), n_layers side layers of height 2 / n_layers, caps
    fanned from their centres: 2 n_poly n_layers + 2 n_poly triangles."""
    ang = np.sort(rng.uniform(0, 2 * np.pi, n_poly))
    rad = rng.uniform(0.6, 1.0, n_poly)
    zs = np.linspace(1.0, -1.0, n_layers + 1)
    V = [(r * np.cos(a), r * np.sin(a), z) for z in zs for a, r in zip(ang, rad)]
    top, bot = len(V), len(V) + 1
    V += [(0.0, 0.0, 1.0), (0.0, 0.0, -1.0)]
    V = np.array(V)
    F = []
    for l in range(n_layers):
        for j in range(n_poly):
            a, b = l * n_poly + j, l * n_poly + (j + 1) % n_poly
            c, d = a + n_poly, b + n_poly
            F.append((a, c, d))
            F.append((a, d, b))
    for j in range(n_poly):
        F.append((top, j, (j + 1) % n_poly))
        F.append((bot, n_layers * n_poly + (j + 1) % n_poly, n_layers * n_poly + j))
    F = np.array(F, dtype=np.int32)
    if signed_volume(V, F) < 0:
        F = F[:, [0, 2, 1]].copy()
    return V, F


def batch_bodies_model(n_bodies=256, t_range=(500, 50000), side_range=(16, 128), spacing_range=(25.0, 100.0),
                       seed=21, height=1.0, offset=1.0e5, joint=True) -> Problem:
    """Batched independent closed bodies: perturbed lat-long spheres and
    extruded star-shaped prisms (alternating), triangle counts log-uniform in
    t_range, each body with its own square station grid (side uniform in
    side_range, spacing uniform in spacing_range) `height` above the ground,
    body b shifted by b x `offset` in x so that no two bodies share a
    position.  Densities U(0.1, 0.5) g/cc, susceptibilities U(0, 0.05) SI;
    z-free vertices, one group per body."""
    rng = np.random.default_rng(seed)
    meshes, rho, chi, grids = [], [], [], []
    for b in range(n_bodies):
        T = float(np.exp(rng.uniform(np.log(t_range[0]), np.log(t_range[1]))))
        side = int(rng.integers(side_range[0], side_range[1] + 1))
        spacing = float(rng.uniform(*spacing_range))
        extent = side * spacing
        radius = rng.uniform(0.1, 0.3) * extent
        depth = radius * rng.uniform(1.3, 2.5)
        if b % 2 == 0:
            n_lon = max(4, int(round(np.sqrt(T))))
            n_lat = max(3, int(round(T / (2 * n_lon))) + 1)
            U, F = latlong_sphere(n_lat, n_lon)
            U = U * (1.0 + rng.normal(0, 0.03, (len(U), 1)))
            V = U * radius
        else:
            n_poly = max(6, int(round(np.sqrt(T / 2))))
            n_layers = max(1, int(round((T - 2 * n_poly) / (2 * n_poly))))
            U, F = star_prism(n_poly, n_layers, rng)
            V = U * np.array([radius, radius, 0.5 * radius])
        cx = b * offset
        V = V + np.array([cx, 0.0, -depth])
        meshes.append((V, F, Z_ONLY))
        rho.append(float(rng.uniform(0.1, 0.5)))
        chi.append(float(rng.uniform(0.0, 0.05)))
        grids.append(station_grid(side, spacing, height, center=(cx, 0.0)))
    st = np.concatenate(grids)
    return Problem("batch", rho, chi, meshes, st, st if joint else None,
                   station_groups=[len(g) for g in grids])
