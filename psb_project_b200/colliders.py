"""Collision objects of the reference (src/Kernel/Collision/*) for
psb_set_colliders: a finite plane, a sphere, a cylinder, a triangle mesh and
height fields. Each object acts after a step's integrator and box walls as
its reference kernel executes; include/psb.h states every object's
behaviour, the reference's quirks included.

The constructors take the arguments of the reference's classes:
  PlaneCollision(A, B, C, D, N, elast)          -> plane(...)
  SphereCollision(origin, radius, elast, container) -> sphere(...)
  CylinderCollision(center, direction, baseRadius, length) -> cylinder(...)
  MeshCollision(faces)                          -> mesh(vertices, triangles)
  Linear/Gaussian/Periodic/Combined_HeightFieldCollision -> height(min, max, terms)
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Optional, Sequence

import numpy as np

PLANE, SPHERE, CYLINDER, MESH, HEIGHT = 1, 2, 3, 4, 5
HEIGHT_LINEAR, HEIGHT_GAUSSIAN, HEIGHT_COSINE = 1, 2, 3
MAX_COLLIDERS = 32


class PsbCollider(ctypes.Structure):
    """psb_collider (include/psb.h)."""
    _fields_ = [("type", ctypes.c_int32), ("container", ctypes.c_int32), ("elast", ctypes.c_float),
                ("count", ctypes.c_int32), ("v", ctypes.c_float * 16), ("data", ctypes.c_void_p)]


@dataclass
class Collider:
    type: int
    v: Sequence[float]
    elast: float = 0.0
    container: bool = True
    data: Optional[np.ndarray] = None      # mesh faces (F, 12) or height terms (T, 6), float32

    def struct(self) -> PsbCollider:
        s = PsbCollider()
        s.type, s.container, s.elast = int(self.type), int(bool(self.container)), float(self.elast)
        vv = [float(x) for x in self.v] + [0.0] * (16 - len(self.v))
        s.v[:] = vv
        if self.data is not None:
            d = np.ascontiguousarray(self.data, np.float32)
            self.data = d
            s.count = d.shape[0]
            s.data = d.ctypes.data
        return s

    def oracle_spec(self):
        """(type, v, elast, container, faces, terms) for oracle.Colliders."""
        faces = self.data if self.type == MESH else None
        terms = None if self.type != HEIGHT else np.asarray(self.data, np.float64)
        return (self.type, list(self.v), self.elast, self.container, faces, terms)


def plane(A, B, C, D, N, elast: float = 0.0) -> Collider:
    """A quad A, B, C, D with normal N (PlaneCollision)."""
    return Collider(PLANE, [*A, *B, *C, *D, *N], elast)


def sphere(origin, radius: float, elast: float = 0.0, container: bool = True) -> Collider:
    """SphereCollision: as its launcher executes, always a container."""
    return Collider(SPHERE, [*origin, radius], elast, container)


def cylinder(center, direction, radius: float, length: float) -> Collider:
    """CylinderCollision: a container, restitution 0.3."""
    return Collider(CYLINDER, [*center, *direction, radius, length], 0.3)


def mesh(vertices, triangles, normals=None) -> Collider:
    """MeshCollision from vertices (V, 3) and triangles (F, 3). Face normals
    default to the unit normals of the counter-clockwise winding."""
    v = np.asarray(vertices, np.float64)
    t = np.asarray(triangles, np.int64)
    a, b, c = v[t[:, 0]], v[t[:, 1]], v[t[:, 2]]
    if normals is None:
        n = np.cross(b - a, c - a)
        n /= np.linalg.norm(n, axis=1, keepdims=True)
    else:
        n = np.asarray(normals, np.float64)
    faces = np.concatenate([a, b, c, n], axis=1).astype(np.float32)
    return Collider(MESH, [], 0.0, True, faces)


def linear(a: float, b: float):
    """h = a x + b z (Linear_HeightField)."""
    return (HEIGHT_LINEAR, a, b, 0.0, 0.0, 0.0)


def gaussian(A: float, x0: float, z0: float, p1: float, p2: float):
    """h = A exp(-((x-x0)^2/(2 p1^2) + (z-z0)^2/(2 p2^2))) (Gaussian_HeightField)."""
    return (HEIGHT_GAUSSIAN, A, x0, z0, p1, p2)


def cosine(A: float, k: float, theta: float, phi: float):
    """h = A cos(k (x cos theta + z sin theta) + phi), one term of Periodic_HeightField."""
    return (HEIGHT_COSINE, A, k, theta, phi, 0.0)


def height(min_, max_, terms, elast: float = 0.0) -> Collider:
    """A height field over the footprint [min, max] in x and z, at height
    min.y + the sum of the terms."""
    d = np.asarray(terms, np.float32).reshape(-1, 6)
    return Collider(HEIGHT, [*min_, *max_], elast, True, d)


def structs(objs: Sequence[Collider]):
    """A psb_collider array for psb_set_colliders (keeps the data alive)."""
    arr = (PsbCollider * max(1, len(objs)))()
    for i, o in enumerate(objs):
        arr[i] = o.struct()
    return arr
