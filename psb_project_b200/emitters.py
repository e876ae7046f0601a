"""Emitters of the reference (src/Kernel/Emitters/*) for psb_add_emitter:
particles appended before a step's neighbour search, one emission per step
while the emitter's emissions are fewer than its duration. include/psb.h
states each type's positions; the defaults below are the reference
constructors' (EmitterBox, EmitterSphere and EmitterCylinder emit once).
"""
from __future__ import annotations

import ctypes
from typing import Sequence

import numpy as np

BOX, SPHERE, CYLINDER, HEART, ELLIPSOID, MESH = 1, 2, 3, 4, 5, 6
MAX_EMITTERS = 16


class PsbEmitter(ctypes.Structure):
    """psb_emitter (include/psb.h)."""
    _fields_ = [("type", ctypes.c_int32), ("duration", ctypes.c_int32), ("count", ctypes.c_int32),
                ("n_faces", ctypes.c_int32), ("particle_radius", ctypes.c_float), ("velocity", ctypes.c_float * 3),
                ("v", ctypes.c_float * 12), ("data", ctypes.c_void_p), ("seed", ctypes.c_uint64)]


class Emitter:
    def __init__(self, type_: int, v: Sequence[float], *, particle_radius: float = 0.0, velocity=(0.0, 0.0, 0.0),
                 duration: int = 1, count: int = 0, faces=None, seed: int = 0):
        self.type, self.v = int(type_), [float(x) for x in v]
        self.particle_radius, self.velocity = float(particle_radius), tuple(float(x) for x in velocity)
        self.duration, self.count, self.seed = int(duration), int(count), int(seed)
        self.faces = None if faces is None else np.ascontiguousarray(faces, np.float32).reshape(-1, 9)

    def struct(self) -> PsbEmitter:
        s = PsbEmitter()
        s.type, s.duration, s.count = self.type, self.duration, self.count
        s.particle_radius = self.particle_radius
        s.velocity[:] = list(self.velocity)
        s.v[:] = self.v + [0.0] * (12 - len(self.v))
        s.seed = self.seed
        if self.faces is not None:
            s.n_faces = self.faces.shape[0]
            s.data = self.faces.ctypes.data
        return s


def box(center, size, particle_radius: float, velocity=(0.0, 0.0, 0.0), duration: int = 1, world=(0.0, 0.0, 0.0)):
    """EmitterBox: a float lattice of step 2 particle_radius over the box."""
    return Emitter(BOX, [*center, *size, *world], particle_radius=particle_radius, velocity=velocity,
                   duration=duration)


def sphere(center, radius: float, particle_radius: float, velocity=(0.0, 0.0, 0.0), duration: int = 1):
    """EmitterSphere: rings in layers of step particle_radius."""
    return Emitter(SPHERE, [*center, radius], particle_radius=particle_radius, velocity=velocity, duration=duration)


def cylinder(center, direction, radius: float, length: float, particle_radius: float, velocity=(0.0, 0.0, 0.0),
             duration: int = 1):
    """EmitterCylinder: rings up to the base radius, layers along y."""
    return Emitter(CYLINDER, [*center, *direction, radius, length], particle_radius=particle_radius,
                   velocity=velocity, duration=duration)


def heart(velocity=(0.0, 0.0, 0.0), duration: int = 1):
    """EmitterGirly: the heart surface sampled on [-3, 3]^3 at 0.02."""
    return Emitter(HEART, [], velocity=velocity, duration=duration)


def ellipsoid(center, a: float, b: float, count: int, velocity=(0.0, 0.0, 0.0), duration: int = 1, seed: int = 0):
    """EmitterElipsoide: `count` random particles per emission."""
    return Emitter(ELLIPSOID, [*center, a, b], velocity=velocity, duration=duration, count=count, seed=seed)


def mesh(vertices, triangles, count: int, velocity=(0.0, 0.0, 0.0), duration: int = 1, seed: int = 0):
    """EmitterMesh: `count` random particles per face per emission."""
    v = np.asarray(vertices, np.float64)
    t = np.asarray(triangles, np.int64)
    faces = np.concatenate([v[t[:, 0]], v[t[:, 1]], v[t[:, 2]]], axis=1)
    return Emitter(MESH, [], velocity=velocity, duration=duration, count=count, faces=faces, seed=seed)


def positions(e: Emitter, emission: int = 0) -> np.ndarray:
    """The positions emission number `emission` produces (host, no GPU)."""
    from .runtime import PsbError, lib
    s = e.struct()
    n = ctypes.c_int64(0)
    rc = lib().psb_emitter_positions(ctypes.byref(s), int(emission), 0, None, ctypes.byref(n))
    if rc != 0:
        raise PsbError(rc, "psb_emitter_positions: bad emitter")
    out = np.empty((n.value, 3), np.float32)
    lib().psb_emitter_positions(ctypes.byref(s), int(emission), n.value, out.ctypes.data_as(ctypes.c_void_p),
                                ctypes.byref(n))
    return out
