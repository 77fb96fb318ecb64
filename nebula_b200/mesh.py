"""Triangle meshes for the SDF builder (host-side helpers; the SDF itself is
built on the GPU by nebula_mpm_set_collider_mesh / nebula_mpm_mesh_sdf).

A mesh is an (n, 12) float32 array, one row per triangle: normal, v0, v1, v2
-- the record order of a binary STL file (loadBinarySTL, src/core/MeshSDF.h:22-43).
"""
from __future__ import annotations

import math
import struct

import numpy as np


def load_binary_stl(path) -> np.ndarray:
    """loadBinarySTL (MeshSDF.h:22-43): 80-byte header, u32 count, then per
    triangle 12 float32 (normal, v0, v1, v2) and a u16 attribute."""
    with open(path, "rb") as f:
        f.read(80)
        (count,) = struct.unpack("<I", f.read(4))
        rec = np.dtype([("f", "<f4", (12,)), ("attr", "<u2")])
        data = np.frombuffer(f.read(count * rec.itemsize), dtype=rec, count=count)
    return np.ascontiguousarray(data["f"], np.float32)


def save_binary_stl(path, tris: np.ndarray) -> None:
    t = np.ascontiguousarray(tris, np.float32).reshape(-1, 12)
    rec = np.zeros(t.shape[0], dtype=[("f", "<f4", (12,)), ("attr", "<u2")])
    rec["f"] = t
    with open(path, "wb") as f:
        f.write(b"nebula_b200 binary STL".ljust(80, b" "))
        f.write(struct.pack("<I", t.shape[0]))
        f.write(rec.tobytes())


def _rotate(q, v):
    w, x, y, z = q
    u = np.array([x, y, z], np.float64)
    v = np.asarray(v, np.float64)
    return v + 2.0 * np.cross(u, np.cross(u, v) + w * v)


def transform_triangles(tris: np.ndarray, translation, rotation=(1.0, 0.0, 0.0, 0.0)) -> np.ndarray:
    """transformTriangles (MeshSDF.h:136-141): normals rotated, vertices rotated
    and translated; rotation is a unit quaternion (w, x, y, z)."""
    t = np.asarray(tris, np.float64).reshape(-1, 4, 3)
    out = np.empty_like(t)
    out[:, 0] = np.array([_rotate(rotation, v) for v in t[:, 0]])
    for k in range(1, 4):
        out[:, k] = np.array([_rotate(rotation, v) for v in t[:, k]]) + np.asarray(translation, np.float64)
    return out.reshape(-1, 12).astype(np.float32)


def _faces_to_tris(verts: np.ndarray, faces: np.ndarray) -> np.ndarray:
    a, b, c = verts[faces[:, 0]], verts[faces[:, 1]], verts[faces[:, 2]]
    n = np.cross(b - a, c - a)
    n /= np.maximum(np.linalg.norm(n, axis=1, keepdims=True), 1e-30)
    return np.concatenate([n, a, b, c], axis=1).astype(np.float32)


def icosphere(center, radius: float, subdivisions: int = 3) -> np.ndarray:
    """A closed sphere mesh with outward normals (20 * 4^subdivisions triangles)."""
    t = (1.0 + math.sqrt(5.0)) / 2.0
    v = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t), (t, 0, -1), (t, 0, 1), (-t, 0, -1),
         (-t, 0, 1)]
    verts = [np.array(p, np.float64) / np.linalg.norm(p) for p in v]
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2), (10, 7, 6), (7, 1, 8), (3, 9, 4),
             (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    for _ in range(subdivisions):
        cache = {}

        def mid(i, j):
            key = (min(i, j), max(i, j))
            if key not in cache:
                m = verts[i] + verts[j]
                verts.append(m / np.linalg.norm(m))
                cache[key] = len(verts) - 1
            return cache[key]

        nf = []
        for a, b, c in faces:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = nf
    V = np.array(verts) * radius + np.asarray(center, np.float64)
    return _faces_to_tris(V, np.array(faces))


def torus(center, major: float, minor: float, n_major: int = 32, n_minor: int = 16) -> np.ndarray:
    """A closed torus around the y axis with outward normals (non-convex)."""
    us = np.linspace(0, 2 * np.pi, n_major, endpoint=False)
    vs = np.linspace(0, 2 * np.pi, n_minor, endpoint=False)
    verts = []
    for u in us:
        for v in vs:
            r = major + minor * np.cos(v)
            verts.append((r * np.cos(u), minor * np.sin(v), r * np.sin(u)))
    V = np.array(verts) + np.asarray(center, np.float64)
    faces = []
    for i in range(n_major):
        for j in range(n_minor):
            a = i * n_minor + j
            b = ((i + 1) % n_major) * n_minor + j
            c = ((i + 1) % n_major) * n_minor + (j + 1) % n_minor
            d = i * n_minor + (j + 1) % n_minor
            faces += [(a, d, c), (a, c, b)]
    return _faces_to_tris(V, np.array(faces))
