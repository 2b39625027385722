"""Synthetic problem inputs and the reference's text formats.

Geometry layouts are the ones the reference reads (src/fileio.h):

* dipoles: one line ``x y z px py pz`` per source (importDipoles, fileio.h:110-131);
* RWG meshes: ``vertices.txt`` (``x y z``), ``faces.txt`` (three 0-based vertex
  indices) and ``rwgs.txt`` (``v0 v1 t+ t-``: the two vertices of the shared
  edge, then the two triangles), fileio.h:134-202;
* plane wave: ``amp polx poly polz khx khy khz k`` (importPlaneWave,
  fileio.h:8-27).

The generators are seeded so that every run, test and benchmark sees the same
problem.  Positions come from numpy's PCG64 generator, not the reference's
``std::random_device``-seeded Mersenne twister (fileio.h:35-36), which is not
reproducible.
"""
from __future__ import annotations

import os
from dataclasses import dataclass, field

import numpy as np


@dataclass
class PlaneWave:
    """Incident plane wave (src/excite.h:6-28)."""

    amplitude: float = 1.0
    pol: tuple = (1.0, 0.0, 0.0)
    khat: tuple = (0.0, 0.0, -1.0)
    wavenum: float = 2.0 * np.pi

    def as_array(self) -> np.ndarray:
        return np.array([self.amplitude, *self.pol, *self.khat, self.wavenum], dtype=np.float64)


@dataclass
class Dipoles:
    pos: np.ndarray  # (N, 3) float64
    mom: np.ndarray  # (N, 3) float64

    @property
    def n(self) -> int:
        return int(self.pos.shape[0])


@dataclass
class RWGMesh:
    vertices: np.ndarray  # (V, 3) float64
    faces: np.ndarray  # (F, 3) int32
    rwgs: np.ndarray  # (E, 4) int32: v0, v1, t+, t-

    @property
    def n(self) -> int:
        return int(self.rwgs.shape[0])


def make_dipoles(n: int, side: float = 4.0, seed: int = 1,
                 moment=(1.0, 0.0, 0.0)) -> Dipoles:
    """``n`` dipoles uniform in the cube [-side/2, side/2]^3, all with one moment."""
    rng = np.random.default_rng(seed)
    pos = rng.uniform(-side / 2.0, side / 2.0, size=(n, 3))
    mom = np.tile(np.asarray(moment, dtype=np.float64), (n, 1))
    return Dipoles(pos=np.ascontiguousarray(pos), mom=np.ascontiguousarray(mom))


def make_icosphere(level: int, radius: float = 1.0) -> RWGMesh:
    """Subdivided icosahedron projected onto a sphere, with its RWG edge list.

    ``level`` subdivisions give 20*4**level faces, 10*4**level + 2 vertices and
    30*4**level edges; every edge of the closed surface carries one RWG function.
    Faces are wound counter-clockwise seen from outside.
    """
    t = (1.0 + 5.0 ** 0.5) / 2.0
    verts = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0),
             (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
             (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    verts = [np.array(v, dtype=np.float64) / np.linalg.norm(v) for v in verts]
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11),
             (1, 5, 9), (5, 11, 4), (11, 10, 2), (10, 7, 6), (7, 1, 8),
             (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9),
             (4, 9, 5), (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    for _ in range(level):
        mid_cache: dict = {}

        def midpoint(a: int, b: int) -> int:
            key = (a, b) if a < b else (b, a)
            if key not in mid_cache:
                m = verts[a] + verts[b]
                verts.append(m / np.linalg.norm(m))
                mid_cache[key] = len(verts) - 1
            return mid_cache[key]

        new_faces = []
        for a, b, c in faces:
            ab, bc, ca = midpoint(a, b), midpoint(b, c), midpoint(c, a)
            new_faces += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = new_faces
    V = np.array(verts) * radius
    F = np.array(faces, dtype=np.int32)
    # Edge -> the two faces sharing it, in face order.
    edge_faces: dict = {}
    for fi, (a, b, c) in enumerate(faces):
        for u, v in ((a, b), (b, c), (c, a)):
            key = (u, v) if u < v else (v, u)
            edge_faces.setdefault(key, []).append(fi)
    rwgs = []
    for (u, v), fs in sorted(edge_faces.items()):
        assert len(fs) == 2, "mesh is not closed"
        rwgs.append((u, v, fs[0], fs[1]))
    return RWGMesh(vertices=np.ascontiguousarray(V), faces=F,
                   rwgs=np.ascontiguousarray(np.array(rwgs, dtype=np.int32)))


# ---------------------------------------------------------------- text formats

def write_dipoles(path: str, d: Dipoles) -> None:
    np.savetxt(path, np.hstack([d.pos, d.mom]), fmt="%.17g")


def read_dipoles(path: str) -> Dipoles:
    a = np.loadtxt(path, dtype=np.float64, ndmin=2)
    if a.shape[1] != 6:
        raise RuntimeError("Unable to parse line")
    return Dipoles(pos=np.ascontiguousarray(a[:, :3]), mom=np.ascontiguousarray(a[:, 3:]))


def write_rwg(directory: str, m: RWGMesh) -> None:
    os.makedirs(directory, exist_ok=True)
    np.savetxt(os.path.join(directory, "vertices.txt"), m.vertices, fmt="%.17g")
    np.savetxt(os.path.join(directory, "faces.txt"), m.faces, fmt="%d")
    np.savetxt(os.path.join(directory, "rwgs.txt"), m.rwgs, fmt="%d")


def read_rwg(directory: str) -> RWGMesh:
    def load(name, dtype, ncol):
        p = os.path.join(directory, name)
        if not os.path.exists(p):
            raise RuntimeError("Unable to find file")
        a = np.loadtxt(p, dtype=dtype, ndmin=2)
        if a.shape[1] != ncol:
            raise RuntimeError("Unable to parse line")
        return np.ascontiguousarray(a)

    return RWGMesh(vertices=load("vertices.txt", np.float64, 3),
                   faces=load("faces.txt", np.int32, 3),
                   rwgs=load("rwgs.txt", np.int32, 4))


def write_planewave(path: str, pw: PlaneWave) -> None:
    with open(path, "w") as f:
        f.write(" ".join("%.17g" % v for v in pw.as_array()) + "\n")


def read_planewave(path: str) -> PlaneWave:
    if not os.path.exists(path):
        raise RuntimeError("Unable to find file")
    with open(path) as f:
        vals = f.readline().split()
    if len(vals) != 8:
        raise RuntimeError("Unable to parse line")
    v = [float(x) for x in vals]
    return PlaneWave(amplitude=v[0], pol=tuple(v[1:4]), khat=tuple(v[4:7]), wavenum=v[7])


def fibonacci_planewaves(n: int, wavenum: float = 2.0 * np.pi, amplitude: float = 1.0) -> list[PlaneWave]:
    """n incident plane waves with directions on a Fibonacci sphere, each
    polarised along theta-hat of its direction (the many-right-hand-side
    benchmark excitation)."""
    golden = np.pi * (3.0 - np.sqrt(5.0))
    out = []
    for i in range(n):
        z = 1.0 - 2.0 * (i + 0.5) / n
        rho = np.sqrt(max(0.0, 1.0 - z * z))
        phi = golden * i
        k = np.array([rho * np.cos(phi), rho * np.sin(phi), z])
        th = np.arccos(np.clip(z, -1.0, 1.0))
        pol = np.array([np.cos(th) * np.cos(phi), np.cos(th) * np.sin(phi), -np.sin(th)])
        out.append(PlaneWave(amplitude=amplitude, pol=tuple(pol), khat=tuple(k), wavenum=wavenum))
    return out
