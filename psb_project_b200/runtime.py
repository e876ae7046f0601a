"""ctypes host API over libpsb.so (include/psb.h).

The library is loaded from this package's lib/ directory, where
``python -m psb_project_b200.build`` (or ``__graft_entry__.build()``) puts it.
There is no fallback: without the compiled library every call raises.
"""
from __future__ import annotations

import ctypes
import os
from typing import Dict, Optional, Tuple

import numpy as np

from .scene import PsbScene, Scene

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libpsb.so")

OK, EINVAL, ENOMEM, EOVERFLOW_NBR, ENOCONV, ECUDA, ESTATE = range(7)
PSB_MAX_ITERS = 64

FIELD_POS, FIELD_VEL, FIELD_VEL_HALF, FIELD_DENSITY, FIELD_PRESSURE, FIELD_DENSITY_X, FIELD_FORCE_NP, \
    FIELD_NBR_COUNT, FIELD_CELL_KEY, FIELD_SORTED_ID, FIELD_SORTED_KEY = range(11)

_FIELD_SPEC: Dict[int, Tuple[type, int]] = {
    FIELD_POS: (np.float32, 3), FIELD_VEL: (np.float32, 3), FIELD_VEL_HALF: (np.float32, 3),
    FIELD_DENSITY: (np.float32, 1), FIELD_PRESSURE: (np.float32, 1), FIELD_DENSITY_X: (np.float32, 1),
    FIELD_FORCE_NP: (np.float32, 3), FIELD_NBR_COUNT: (np.int32, 1), FIELD_CELL_KEY: (np.uint32, 1),
    FIELD_SORTED_ID: (np.int32, 1), FIELD_SORTED_KEY: (np.uint32, 1),
}

# Every symbol include/psb.h declares (the tests check the library exports all of them).
EXPORTS = (
    "psb_create", "psb_destroy", "psb_set_stream", "psb_upload", "psb_upload_aos_f64", "psb_download",
    "psb_download_aos_f64", "psb_step", "psb_build_neighbors", "psb_read_field", "psb_get_stats",
    "psb_profile_enable", "psb_profile_read", "psb_profile_reset", "psb_lattice", "psb_status_string",
    "psb_last_error", "psb_abi_version", "psb_sort_cells_noalloc", "psb_presolve", "psb_mlp_set_weights",
    "psb_mlp_get_weights", "psb_mlp_collect", "psb_mlp_dataset", "psb_mlp_train", "psb_mlp_forward",
    "psb_mlp_loss_grad", "psb_iso_field", "psb_extract_surface", "psb_create_batch", "psb_batch_layout",
    "psb_batch_stats", "psb_set_graph", "psb_set_corrector", "psb_autotune", "psb_tune_set", "psb_tune_get", "psb_diagnostics",
    "psb_set_boundary", "psb_boundary_psi", "psb_context_info", "psb_set_step_count", "psb_write_txt",
    "psb_write_xml", "psb_write_vol", "psb_write_obj", "psb_export_txt", "psb_export_xml", "psb_checkpoint_save",
    "psb_checkpoint_load", "psb_boundary_forces", "psb_set_external_force", "psb_set_colliders", "psb_emit",
    "psb_add_emitter", "psb_clear_emitters", "psb_emitter_positions", "psb_mlp_set_arch", "psb_mlp_info",
    "psb_warm_start", "psb_set_boundary_motion", "psb_dem_forces",
)
MLP_SILU6, MLP_RELU7 = 0, 1   # PSB_MLP_SILU6 (the configured network), PSB_MLP_RELU7
CORRECTOR_LAUNCHES, CORRECTOR_PERSISTENT = 0, 1   # PSB_CORRECTOR_*
MLP_PARAMS = 4737       # PSB_MLP_PARAMS: the larger network's count
MLP_H = 64
MLP_INPUTS = {MLP_SILU6: 6, MLP_RELU7: 7}
NOALLOC_MAX_N = 262144   # PSB_NOALLOC_MAX_N


class PsbStepStats(ctypes.Structure):
    _fields_ = [
        ("iters", ctypes.c_int32), ("converged", ctypes.c_int32), ("nbr_max", ctypes.c_int32),
        ("clamped", ctypes.c_int32), ("nbr_total", ctypes.c_int64),
        ("err", ctypes.c_double * (PSB_MAX_ITERS + 1)), ("steps", ctypes.c_int64), ("iters_total", ctypes.c_int64),
    ]


class PsbTune(ctypes.Structure):
    """psb_tune: the autotuner's launch configuration for one size bucket."""
    _fields_ = [("bucket", ctypes.c_int32), ("nbr_block", ctypes.c_int32), ("nbr_schedule", ctypes.c_int32),
                ("density_block", ctypes.c_int32), ("init_block", ctypes.c_int32),
                ("pci_density_block", ctypes.c_int32), ("force_block", ctypes.c_int32),
                ("xsph_block", ctypes.c_int32), ("ms", ctypes.c_double * 6), ("ms_default", ctypes.c_double * 6)]

    KERNELS = ("build_nbr", "density_x", "pci_init", "pci_density", "pci_force_predict", "xsph")

    def as_dict(self) -> dict:
        d = {k: getattr(self, k) for k, _ in self._fields_[:8]}
        d["ms"] = dict(zip(self.KERNELS, list(self.ms)))
        d["ms_default"] = dict(zip(self.KERNELS, list(self.ms_default)))
        return d


class PsbDiag(ctypes.Structure):
    """psb_diag: FP64 mass, momentum and energy of the current state."""
    _fields_ = [("mass", ctypes.c_double), ("momentum", ctypes.c_double * 3), ("kinetic", ctypes.c_double),
                ("potential", ctypes.c_double), ("density_err_mean", ctypes.c_double),
                ("density_err_max", ctypes.c_double)]

    def as_dict(self) -> dict:
        return {"mass": self.mass, "momentum": list(self.momentum), "kinetic": self.kinetic,
                "potential": self.potential, "density_err_mean": self.density_err_mean,
                "density_err_max": self.density_err_max}


class IsoGrid(ctypes.Structure):
    """psb_iso_grid: dims[a] nodes along axis a at origin[a] + i spacing[a], x fastest."""
    _fields_ = [("origin", ctypes.c_double * 3), ("spacing", ctypes.c_double * 3), ("dims", ctypes.c_int32 * 3),
                ("scale", ctypes.c_double)]


def iso_grid(origin, spacing, dims, scale: float = 0.65) -> IsoGrid:
    """A node grid; `spacing` is one value or one per axis. `scale` is the
    reference profile's influence-radius divisor (SurfaceSPH::extract: 0.65)."""
    g = IsoGrid()
    g.origin[:] = [float(v) for v in origin]
    sp = spacing if hasattr(spacing, "__len__") else (spacing,) * 3
    g.spacing[:] = [float(v) for v in sp]
    g.dims[:] = [int(v) for v in dims]
    g.scale = float(scale)
    return g


class PsbError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"[{status}] {message}")
        self.status = status


_lib = None


def lib():
    """The loaded libpsb.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m psb_project_b200.build`")
    L = ctypes.CDLL(LIB_PATH)
    P, I32, I64 = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64
    sig = {
        "psb_create": ([ctypes.POINTER(PsbScene), ctypes.POINTER(P)], ctypes.c_int),
        "psb_destroy": ([P], ctypes.c_int),
        "psb_set_stream": ([P, P], ctypes.c_int),
        "psb_upload": ([P, I32, P, P, P, P], ctypes.c_int),
        "psb_upload_aos_f64": ([P, I32, P, P, P, I32], ctypes.c_int),
        "psb_download": ([P, P, P, P, P, P], ctypes.c_int),
        "psb_download_aos_f64": ([P, P, P, P, I32], ctypes.c_int),
        "psb_step": ([P, I32], ctypes.c_int),
        "psb_build_neighbors": ([P], ctypes.c_int),
        "psb_read_field": ([P, I32, P, ctypes.c_size_t], ctypes.c_int),
        "psb_get_stats": ([P, ctypes.POINTER(PsbStepStats)], ctypes.c_int),
        "psb_profile_enable": ([P, I32], ctypes.c_int),
        "psb_profile_read": ([P, I32, ctypes.c_char_p, ctypes.c_size_t, ctypes.POINTER(I64),
                              ctypes.POINTER(ctypes.c_double)], ctypes.c_int),
        "psb_profile_reset": ([P], ctypes.c_int),
        "psb_lattice": ([P, ctypes.c_double, P, ctypes.c_double, ctypes.c_uint64, I32, P], ctypes.c_int),
        "psb_status_string": ([I32], ctypes.c_char_p),
        "psb_last_error": ([P], ctypes.c_char_p),
        "psb_abi_version": ([], I32),
        "psb_sort_cells_noalloc": ([P, P, P, P, I32, I32, P], ctypes.c_int),
        "psb_presolve": ([P, I32], ctypes.c_int),
        "psb_mlp_set_weights": ([P, P], ctypes.c_int),
        "psb_mlp_set_arch": ([P, I32], ctypes.c_int),
        "psb_mlp_info": ([P, P, P, P], ctypes.c_int),
        "psb_warm_start": ([P, P, P], ctypes.c_int),
        "psb_mlp_get_weights": ([P, P], ctypes.c_int),
        "psb_mlp_collect": ([P, I32, I64], ctypes.c_int),
        "psb_mlp_dataset": ([P, ctypes.POINTER(I64), P, P], ctypes.c_int),
        "psb_mlp_train": ([P, I32, I32, ctypes.c_float, ctypes.c_uint64, ctypes.POINTER(ctypes.c_float)], ctypes.c_int),
        "psb_mlp_forward": ([P, P, I32, P], ctypes.c_int),
        "psb_mlp_loss_grad": ([P, P, P, I32, ctypes.POINTER(ctypes.c_float), P], ctypes.c_int),
        "psb_iso_field": ([P, ctypes.POINTER(IsoGrid), P], ctypes.c_int),
        "psb_extract_surface": ([P, ctypes.POINTER(IsoGrid), ctypes.c_double, P, ctypes.POINTER(I64), P,
                                 ctypes.POINTER(I64)], ctypes.c_int),
        "psb_create_batch": ([ctypes.POINTER(PsbScene), I32, ctypes.POINTER(P)], ctypes.c_int),
        "psb_batch_layout": ([P, ctypes.POINTER(I32), P], ctypes.c_int),
        "psb_batch_stats": ([P, P, P, P, P, P], ctypes.c_int),
        "psb_set_graph": ([P, I32], ctypes.c_int),
        "psb_set_corrector": ([P, I32], ctypes.c_int),
        "psb_autotune": ([P, I32, ctypes.POINTER(PsbTune)], ctypes.c_int),
        "psb_tune_set": ([P, ctypes.POINTER(PsbTune)], ctypes.c_int),
        "psb_tune_get": ([P, I32, ctypes.POINTER(PsbTune)], ctypes.c_int),
        "psb_diagnostics": ([P, ctypes.POINTER(PsbDiag), I32], ctypes.c_int),
        "psb_set_boundary": ([P, I32, P], ctypes.c_int),
        "psb_boundary_psi": ([P, P], ctypes.c_int),
        "psb_context_info": ([P, ctypes.POINTER(PsbScene), ctypes.POINTER(I32), ctypes.POINTER(I64)], ctypes.c_int),
        "psb_set_step_count": ([P, I64], ctypes.c_int),
        "psb_write_txt": ([ctypes.c_char_p, I32, P, ctypes.c_double, P], ctypes.c_int),
        "psb_write_xml": ([ctypes.c_char_p, ctypes.POINTER(PsbScene), I32, P, P, P, P], ctypes.c_int),
        "psb_write_vol": ([ctypes.c_char_p, P, P, P, P, I32], ctypes.c_int),
        "psb_write_obj": ([ctypes.c_char_p, P, I64, P, I64], ctypes.c_int),
        "psb_export_txt": ([P, ctypes.c_char_p], ctypes.c_int),
        "psb_export_xml": ([P, ctypes.c_char_p], ctypes.c_int),
        "psb_checkpoint_save": ([P, ctypes.c_char_p], ctypes.c_int),
        "psb_checkpoint_load": ([P, ctypes.c_char_p], ctypes.c_int),
        "psb_boundary_forces": ([P, P], ctypes.c_int),
        "psb_set_external_force": ([P, P], ctypes.c_int),
        "psb_set_boundary_motion": ([P, P, P, ctypes.c_float], ctypes.c_int),
        "psb_dem_forces": ([P, P], ctypes.c_int),
        "psb_set_colliders": ([P, P, I32], ctypes.c_int),
        "psb_emit": ([P, I32, P, P, P], ctypes.c_int),
        "psb_add_emitter": ([P, P], ctypes.c_int),
        "psb_clear_emitters": ([P], ctypes.c_int),
        "psb_emitter_positions": ([P, I32, ctypes.c_int64, P, P], ctypes.c_int),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    _lib = L
    return L


def _ptr(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def lattice(nxyz, spacing, origin, jitter, seed, id0=0) -> np.ndarray:
    """Lattice block positions (float32, (n, 3), ids x-fastest)."""
    n = int(nxyz[0]) * int(nxyz[1]) * int(nxyz[2])
    out = np.empty((n, 3), np.float32)
    nx = np.asarray(nxyz, np.int32)
    org = np.asarray(origin, np.float64)
    rc = lib().psb_lattice(_ptr(nx), float(spacing), _ptr(org), float(jitter), int(seed) & (2**64 - 1), int(id0),
                           _ptr(out))
    if rc != OK:
        raise PsbError(rc, "psb_lattice")
    return out


def mlp_params(arch: int = MLP_SILU6) -> int:
    """Parameter count of a network: 64 n_in + 64 + 64 x 64 + 64 + 64 + 1."""
    return MLP_H * MLP_INPUTS[arch] + MLP_H + MLP_H * MLP_H + MLP_H + MLP_H + 1


def mlp_init_weights(seed: int = 0, arch: int = MLP_SILU6) -> np.ndarray:
    """He-uniform initial weights in the psb_mlp layout: W1[64][n_in], b1[64],
    W2[64][64], b2[64], W3[64], b3 (biases zero)."""
    rng = np.random.default_rng(seed)
    w = np.zeros(mlp_params(arch), np.float32)
    o = 0
    for fan_in, fan_out in ((MLP_INPUTS[arch], MLP_H), (MLP_H, MLP_H), (MLP_H, 1)):
        lim = np.sqrt(6.0 / fan_in)
        w[o:o + fan_in * fan_out] = rng.uniform(-lim, lim, fan_in * fan_out) * (0.5 if fan_out == 1 else 1.0)
        o += fan_in * fan_out + fan_out
    return w


def mlp_unpack(w: np.ndarray):
    """(W1, b1, W2, b2, W3, b3) views of a flat parameter vector (either
    network: the input count follows from the length)."""
    n_in = (len(w) - (MLP_H + MLP_H * MLP_H + MLP_H + MLP_H + 1)) // MLP_H
    o = 0
    out = []
    for shape in ((MLP_H, n_in), (MLP_H,), (MLP_H, MLP_H), (MLP_H,), (MLP_H,), (1,)):
        k = int(np.prod(shape))
        out.append(w[o:o + k].reshape(shape))
        o += k
    return out


def _status(rc: int, what: str):
    if rc != OK:
        raise PsbError(rc, f"{what}: {lib().psb_status_string(rc).decode()}")


def write_txt(path: str, pos, mass: float, density):
    """Txt particle file (the reference's ParticleExporter_Txt format)."""
    pos = np.ascontiguousarray(pos, np.float64).reshape(-1, 3)
    rho = np.ascontiguousarray(density, np.float32)
    _status(lib().psb_write_txt(path.encode(), pos.shape[0], _ptr(pos), float(mass), _ptr(rho)), "psb_write_txt")


def write_xml(path: str, scene: Scene, pos, vel, vel_half, nbr_count=None):
    """XML particle file (the reference's ParticleExporter_XML SPH format)."""
    cv = lambda a: np.ascontiguousarray(a, np.float64).reshape(-1, 3)
    pos, vel, vel_half = cv(pos), cv(vel), cv(vel_half)
    nb = None if nbr_count is None else np.ascontiguousarray(nbr_count, np.int32)
    sc = scene.to_c()
    _status(lib().psb_write_xml(path.encode(), ctypes.byref(sc), pos.shape[0], _ptr(pos), _ptr(vel), _ptr(vel_half),
                                _ptr(nb)), "psb_write_xml")


def write_vol(path: str, field, dims, bmin, bmax, reference_layout: bool = False):
    """Mitsuba grid volume of a node field (x fastest, as iso_field returns it)."""
    f = np.ascontiguousarray(field, np.float64)
    d = np.asarray(dims, np.int32)
    lo = np.asarray(bmin, np.float32)
    hi = np.asarray(bmax, np.float32)
    _status(lib().psb_write_vol(path.encode(), _ptr(f), _ptr(d), _ptr(lo), _ptr(hi), 1 if reference_layout else 0),
            "psb_write_vol")


def write_obj(path: str, vertices, triangles):
    """Wavefront OBJ of a triangle mesh, with area-weighted vertex normals."""
    v = np.ascontiguousarray(vertices, np.float32).reshape(-1, 3)
    t = np.ascontiguousarray(triangles, np.int32).reshape(-1, 3)
    _status(lib().psb_write_obj(path.encode(), _ptr(v), v.shape[0], _ptr(t), t.shape[0]), "psb_write_obj")


def scene_positions(scene: Scene) -> np.ndarray:
    return np.concatenate([lattice(b.nxyz, b.spacing, b.origin, b.jitter, b.seed, b.id0) for b in scene.blocks])


class Simulation:
    """One psb_ctx: a scene's particles resident in HBM, stepped on a stream."""

    def __init__(self, scene: Scene):
        self.scene = scene
        self._c = scene.to_c()
        h = ctypes.c_void_p()
        rc = lib().psb_create(ctypes.byref(self._c), ctypes.byref(h))
        if rc != OK:
            raise PsbError(rc, f"psb_create: {lib().psb_status_string(rc).decode()}")
        self._h = h
        self.n = 0

    # -- lifecycle ------------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None):
            lib().psb_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, rc: int, what: str, allow=(OK,)):
        if rc not in allow:
            msg = lib().psb_last_error(self._h)
            raise PsbError(rc, f"{what}: {lib().psb_status_string(rc).decode()}: {msg.decode() if msg else ''}")
        return rc

    # -- calls ----------------------------------------------------------------
    def set_stream(self, stream_ptr: int):
        self._check(lib().psb_set_stream(self._h, ctypes.c_void_p(stream_ptr)), "psb_set_stream")

    def upload(self, pos, vel=None, vel_half=None, pressure=None):
        pos = np.ascontiguousarray(pos, np.float32)
        n = pos.shape[0]
        cv = lambda a: None if a is None else np.ascontiguousarray(a, np.float32)
        vel, vel_half, pressure = cv(vel), cv(vel_half), cv(pressure)
        self._check(lib().psb_upload(self._h, n, _ptr(pos), _ptr(vel), _ptr(vel_half), _ptr(pressure)), "psb_upload")
        self.n = n

    def upload_aos_f64(self, pos, vel=None, vel_half=None, on_device=False):
        if on_device:
            p = lambda a: None if a is None else ctypes.c_void_p(int(a))
            rc = lib().psb_upload_aos_f64(self._h, self.scene.n if self.n == 0 else self.n, p(pos), p(vel), p(vel_half), 1)
            self._check(rc, "psb_upload_aos_f64")
            return
        pos = np.ascontiguousarray(pos, np.float64)
        cv = lambda a: None if a is None else np.ascontiguousarray(a, np.float64)
        vel, vel_half = cv(vel), cv(vel_half)
        self._check(lib().psb_upload_aos_f64(self._h, pos.shape[0], _ptr(pos), _ptr(vel), _ptr(vel_half), 0),
                    "psb_upload_aos_f64")
        self.n = pos.shape[0]

    def step(self, nsteps: int = 1, allow_noconv: bool = True) -> int:
        allow = (OK, ENOCONV) if allow_noconv else (OK,)
        rc = lib().psb_step(self._h, int(nsteps))
        if getattr(self, "_emitting", False):      # emitters grow the particle count inside the step
            n = ctypes.c_int32()
            lib().psb_context_info(self._h, None, ctypes.byref(n), None)
            self.n = n.value
        return self._check(rc, "psb_step", allow)

    def presolve(self, iters: int):
        self._check(lib().psb_presolve(self._h, int(iters)), "psb_presolve")

    # -- learned warm start -------------------------------------------------------
    def mlp_set_arch(self, arch: int):
        """Selects the network (MLP_SILU6, the configured one and the default,
        or MLP_RELU7); clears its weights."""
        self._check(lib().psb_mlp_set_arch(self._h, int(arch)), "psb_mlp_set_arch")

    def mlp_info(self) -> dict:
        a, ni, npar = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
        self._check(lib().psb_mlp_info(self._h, ctypes.byref(a), ctypes.byref(ni), ctypes.byref(npar)), "psb_mlp_info")
        return {"arch": a.value, "n_inputs": ni.value, "n_params": npar.value}

    def mlp_set_weights(self, w):
        w = np.ascontiguousarray(w, np.float32)
        if w.shape != (self.mlp_info()["n_params"],):
            raise ValueError(f"weights of shape {w.shape} for a network of {self.mlp_info()['n_params']} parameters")
        self._check(lib().psb_mlp_set_weights(self._h, _ptr(w)), "psb_mlp_set_weights")

    def mlp_get_weights(self) -> np.ndarray:
        w = np.empty(self.mlp_info()["n_params"], np.float32)
        self._check(lib().psb_mlp_get_weights(self._h, _ptr(w)), "psb_mlp_get_weights")
        return w

    def warm_start(self):
        """(features (n, 8), initial pressure (n,)) of the next step, id
        order, without stepping (psb_warm_start)."""
        n = self.n
        F = np.empty((n, 8), np.float32)
        p = np.empty(n, np.float32)
        self._check(lib().psb_warm_start(self._h, _ptr(F), _ptr(p)), "psb_warm_start")
        return F, p

    def mlp_collect(self, stride: int, capacity: int = 1 << 22):
        self._check(lib().psb_mlp_collect(self._h, int(stride), int(capacity)), "psb_mlp_collect")

    def mlp_dataset(self, fetch: bool = True):
        rows = ctypes.c_int64()
        self._check(lib().psb_mlp_dataset(self._h, ctypes.byref(rows), None, None), "psb_mlp_dataset")
        if not fetch:
            return rows.value, None, None
        X = np.empty((rows.value, 8), np.float32)
        T = np.empty(rows.value, np.float32)
        self._check(lib().psb_mlp_dataset(self._h, ctypes.byref(rows), _ptr(X), _ptr(T)), "psb_mlp_dataset")
        return rows.value, X, T

    def mlp_train(self, iters: int, batch: int, lr: float, seed: int = 0) -> float:
        loss = ctypes.c_float()
        self._check(lib().psb_mlp_train(self._h, int(iters), int(batch), float(lr), int(seed), ctypes.byref(loss)),
                    "psb_mlp_train")
        return loss.value

    def mlp_fit(self, iters: int, batch: int, lr: float, chunks: int = 10, seed: int = 0) -> float:
        """Adam on the collected pairs with a cosine-decayed learning rate:
        `chunks` equal runs of psb_mlp_train, the k-th at
        lr * (1 + cos(pi (k + 1/2) / chunks)) / 2. Adam's moments carry over
        between the chunks. Returns the last chunk's loss."""
        loss = float("nan")
        for k in range(chunks):
            lr_k = lr * 0.5 * (1.0 + np.cos(np.pi * (k + 0.5) / chunks))
            loss = self.mlp_train(max(1, iters // chunks), batch, lr_k, seed=seed * 1000 + k)
        return loss

    def mlp_forward(self, X) -> np.ndarray:
        X8 = np.zeros((X.shape[0], 8), np.float32)
        X8[:, :X.shape[1]] = X
        y = np.empty(X.shape[0], np.float32)
        self._check(lib().psb_mlp_forward(self._h, _ptr(X8), X.shape[0], _ptr(y)), "psb_mlp_forward")
        return y

    def mlp_loss_grad(self, X, T):
        X8 = np.zeros((X.shape[0], 8), np.float32)
        X8[:, :X.shape[1]] = X
        T = np.ascontiguousarray(T, np.float32)
        g = np.empty(self.mlp_info()["n_params"], np.float32)
        loss = ctypes.c_float()
        self._check(lib().psb_mlp_loss_grad(self._h, _ptr(X8), _ptr(T), X.shape[0], ctypes.byref(loss), _ptr(g)),
                    "psb_mlp_loss_grad")
        return loss.value, g

    def build_neighbors(self):
        self._check(lib().psb_build_neighbors(self._h), "psb_build_neighbors")

    def iso_field(self, grid: IsoGrid) -> np.ndarray:
        """psb_iso_field: the field at every node (x fastest), float64."""
        out = np.empty(int(grid.dims[0]) * int(grid.dims[1]) * int(grid.dims[2]), np.float64)
        self._check(lib().psb_iso_field(self._h, ctypes.byref(grid), _ptr(out)), "psb_iso_field")
        return out

    def extract_surface(self, grid: IsoGrid, level: float):
        """psb_extract_surface: (vertices (V, 3) float32, triangles (T, 3) int32)."""
        nv = ctypes.c_int64(0)
        nt = ctypes.c_int64(0)
        self._check(lib().psb_extract_surface(self._h, ctypes.byref(grid), float(level), None, ctypes.byref(nv), None,
                                              ctypes.byref(nt)), "psb_extract_surface")
        vert = np.empty((max(nv.value, 1), 3), np.float32)
        tri = np.empty((max(nt.value, 1), 3), np.int32)
        self._check(lib().psb_extract_surface(self._h, ctypes.byref(grid), float(level), _ptr(vert), ctypes.byref(nv),
                                              _ptr(tri), ctypes.byref(nt)), "psb_extract_surface")
        return vert[:nv.value], tri[:nt.value]

    def extract_surface_into(self, grid: IsoGrid, level: float, vert: np.ndarray, tri: np.ndarray):
        """psb_extract_surface in one call into caller buffers (vert (V, 3)
        float32, tri (T, 3) int32, both C-contiguous); returns (V, T) used."""
        nv = ctypes.c_int64(vert.shape[0])
        nt = ctypes.c_int64(tri.shape[0])
        self._check(lib().psb_extract_surface(self._h, ctypes.byref(grid), float(level), _ptr(vert), ctypes.byref(nv),
                                              _ptr(tri), ctypes.byref(nt)), "psb_extract_surface")
        return nv.value, nt.value

    def download(self, out: Optional[dict] = None) -> dict:
        n = self.n
        o = out if out is not None else {
            "pos": np.empty((n, 3), np.float32), "vel": np.empty((n, 3), np.float32),
            "vel_half": np.empty((n, 3), np.float32), "density": np.empty(n, np.float32),
            "pressure": np.empty(n, np.float32)}
        self._check(lib().psb_download(self._h, _ptr(o.get("pos")), _ptr(o.get("vel")), _ptr(o.get("vel_half")),
                                       _ptr(o.get("density")), _ptr(o.get("pressure"))), "psb_download")
        return o

    def download_aos_f64(self) -> dict:
        n = self.n
        o = {k: np.empty((n, 3), np.float64) for k in ("pos", "vel", "vel_half")}
        self._check(lib().psb_download_aos_f64(self._h, _ptr(o["pos"]), _ptr(o["vel"]), _ptr(o["vel_half"]), 0),
                    "psb_download_aos_f64")
        return o

    def read_field(self, field: int) -> np.ndarray:
        dt, w = _FIELD_SPEC[field]
        out = np.empty((self.n, w) if w > 1 else self.n, dt)
        self._check(lib().psb_read_field(self._h, field, _ptr(out), out.nbytes), "psb_read_field")
        return out

    def stats(self) -> PsbStepStats:
        s = PsbStepStats()
        self._check(lib().psb_get_stats(self._h, ctypes.byref(s)), "psb_get_stats")
        return s

    # -- boundary particles ------------------------------------------------------
    def set_boundary(self, pos):
        """Static boundary particles (config profile): positions (n_b, 3)."""
        pos = np.ascontiguousarray(pos, np.float32).reshape(-1, 3)
        self._check(lib().psb_set_boundary(self._h, pos.shape[0], _ptr(pos) if pos.shape[0] else None),
                    "psb_set_boundary")
        self.n_bnd = pos.shape[0]

    def boundary_forces(self) -> np.ndarray:
        """The fluid's force (N) on each boundary particle after the last step, (n_b, 3)."""
        out = np.empty((self.n_bnd, 3), np.float32)
        self._check(lib().psb_boundary_forces(self._h, _ptr(out)), "psb_boundary_forces")
        return out

    def set_boundary_motion(self, vel, force=None, mass: float = 0.0):
        """The boundary set moves with the pressure corrector (config PCISPH):
        velocities and non-fluid forces (n_b, 3) at the step's start and the
        particles' mass; vel None makes it static again."""
        if vel is None:
            self._check(lib().psb_set_boundary_motion(self._h, None, None, 0.0), "psb_set_boundary_motion")
            return
        v = np.ascontiguousarray(vel, np.float32).reshape(-1, 3)
        f = np.ascontiguousarray(force, np.float32).reshape(-1, 3)
        self._check(lib().psb_set_boundary_motion(self._h, _ptr(v), _ptr(f), float(mass)), "psb_set_boundary_motion")

    def dem_forces(self) -> np.ndarray:
        """DEM: gravity and contact force (n, 3) on each sphere at the current state, id order."""
        out = np.empty((self.n, 3), np.float32)
        self._check(lib().psb_dem_forces(self._h, _ptr(out)), "psb_dem_forces")
        return out

    def set_external_force(self, force):
        """DEM: external force per sphere (n, 3) in N, id order; None removes it."""
        if force is None:
            self._check(lib().psb_set_external_force(self._h, None), "psb_set_external_force")
            return
        f = np.ascontiguousarray(force, np.float32).reshape(-1, 3)
        self._check(lib().psb_set_external_force(self._h, _ptr(f)), "psb_set_external_force")

    # -- emission -----------------------------------------------------------------
    def emit(self, pos, vel=None, vel_half=None):
        """Appends particles (ids n .. n + k - 1) to the resident state."""
        pos = np.ascontiguousarray(pos, np.float32).reshape(-1, 3)
        arrs = [None if a is None else np.ascontiguousarray(a, np.float32).reshape(-1, 3) for a in (vel, vel_half)]
        self._check(lib().psb_emit(self._h, pos.shape[0], _ptr(pos), *[None if a is None else _ptr(a) for a in arrs]),
                    "psb_emit")
        self.n += pos.shape[0]

    def add_emitter(self, e):
        """An emitter (psb_project_b200.emitters) that runs inside step()."""
        s = e.struct()
        self._check(lib().psb_add_emitter(self._h, ctypes.byref(s)), "psb_add_emitter")
        self._emitting = True

    def clear_emitters(self):
        self._check(lib().psb_clear_emitters(self._h), "psb_clear_emitters")
        self._emitting = False

    # -- collision objects --------------------------------------------------------
    def set_colliders(self, objs):
        """Collision objects (psb_project_b200.colliders), applied in order
        after each step's box walls; [] removes them."""
        from . import colliders as C
        objs = list(objs)
        arr = C.structs(objs)
        self._check(lib().psb_set_colliders(self._h, ctypes.cast(arr, ctypes.c_void_p) if objs else None, len(objs)),
                    "psb_set_colliders")
        self._colliders = objs

    def boundary_psi(self) -> np.ndarray:
        out = np.empty(self.n_bnd, np.float32)
        self._check(lib().psb_boundary_psi(self._h, _ptr(out)), "psb_boundary_psi")
        return out

    # -- files -------------------------------------------------------------------
    def export_txt(self, path: str):
        self._check(lib().psb_export_txt(self._h, path.encode()), "psb_export_txt")

    def export_xml(self, path: str):
        self._check(lib().psb_export_xml(self._h, path.encode()), "psb_export_xml")

    def checkpoint_save(self, path: str):
        self._check(lib().psb_checkpoint_save(self._h, path.encode()), "psb_checkpoint_save")

    def checkpoint_load(self, path: str):
        self._check(lib().psb_checkpoint_load(self._h, path.encode()), "psb_checkpoint_load")
        n = ctypes.c_int32()
        self._check(lib().psb_context_info(self._h, None, ctypes.byref(n), None), "psb_context_info")
        self.n = n.value

    def steps_taken(self) -> int:
        st = ctypes.c_int64()
        self._check(lib().psb_context_info(self._h, None, None, ctypes.byref(st)), "psb_context_info")
        return st.value

    # -- diagnostics -------------------------------------------------------------
    def diagnostics(self, per_scene: bool = False):
        """FP64 mass, momentum, energies and density-error statistics (a list
        with one dict per scene when per_scene, else one dict)."""
        k = len(getattr(self, "scenes", [None])) if per_scene else 1
        arr = (PsbDiag * k)()
        self._check(lib().psb_diagnostics(self._h, arr, k), "psb_diagnostics")
        out = [d.as_dict() for d in arr]
        return out if per_scene else out[0]

    # -- autotuner ---------------------------------------------------------------
    def autotune(self, trials: int = 5) -> dict:
        """Times the launch configurations on the current particles (after a
        step) and keeps the fastest for this particle count's size bucket."""
        t = PsbTune()
        self._check(lib().psb_autotune(self._h, int(trials), ctypes.byref(t)), "psb_autotune")
        return t.as_dict()

    def tune_set(self, bucket: int, nbr_block=0, nbr_schedule=0, density_block=0, init_block=0,
                 pci_density_block=0, force_block=0, xsph_block=0):
        t = PsbTune(bucket=bucket, nbr_block=nbr_block, nbr_schedule=nbr_schedule, density_block=density_block,
                    init_block=init_block, pci_density_block=pci_density_block, force_block=force_block,
                    xsph_block=xsph_block)
        self._check(lib().psb_tune_set(self._h, ctypes.byref(t)), "psb_tune_set")

    def tune_get(self, bucket: int) -> dict:
        t = PsbTune()
        self._check(lib().psb_tune_get(self._h, int(bucket), ctypes.byref(t)), "psb_tune_get")
        return t.as_dict()

    @staticmethod
    def size_bucket(n: int) -> int:
        return int(n).bit_length() - 1

    TUNE_FIELDS = ("nbr_block", "nbr_schedule", "density_block", "init_block", "pci_density_block", "force_block",
                   "xsph_block")

    def save_tune(self, path: str):
        """Merges this context's tuned buckets into the JSON cache at `path`
        ({bucket: {field: value}}), keeping the other buckets' entries."""
        import json
        table = {}
        if os.path.exists(path):
            with open(path) as f:
                table = json.load(f)
        for b in range(63):
            t = self.tune_get(b)
            if any(t[k] for k in self.TUNE_FIELDS):
                table[str(b)] = {k: int(t[k]) for k in self.TUNE_FIELDS}
        with open(path, "w") as f:
            json.dump(table, f, indent=1, sort_keys=True)

    def load_tune(self, path: str) -> int:
        """Installs every bucket of the JSON cache at `path`; returns how many."""
        import json
        with open(path) as f:
            table = json.load(f)
        for b, e in table.items():
            self.tune_set(int(b), **{k: int(e.get(k, 0)) for k in self.TUNE_FIELDS})
        return len(table)

    def profile(self, on: bool = True):
        self._check(lib().psb_profile_enable(self._h, 1 if on else 0), "psb_profile_enable")

    def set_graph(self, on: bool = True):
        """CUDA-graph stepping (batches and config-profile PCISPH scenes): each
        step one cudaGraphLaunch, the corrector a device-side while loop."""
        self._check(lib().psb_set_graph(self._h, 1 if on else 0), "psb_set_graph")

    def set_corrector(self, mode: int = CORRECTOR_PERSISTENT):
        """The corrector loop (batches and config-profile PCISPH scenes):
        CORRECTOR_LAUNCHES, three kernels per correction, or
        CORRECTOR_PERSISTENT, the whole loop in one cooperative launch."""
        self._check(lib().psb_set_corrector(self._h, int(mode)), "psb_set_corrector")

    def profile_reset(self):
        self._check(lib().psb_profile_reset(self._h), "psb_profile_reset")

    def profile_read(self) -> Dict[str, Tuple[int, float]]:
        res = {}
        i = 0
        buf = ctypes.create_string_buffer(64)
        while True:
            la = ctypes.c_int64()
            ms = ctypes.c_double()
            if lib().psb_profile_read(self._h, i, buf, 64, ctypes.byref(la), ctypes.byref(ms)) != OK:
                break
            res[buf.value.decode()] = (la.value, ms.value)
            i += 1
        return res


class BatchSimulation(Simulation):
    """One psb_ctx over many independent scenes (psb_create_batch): every
    sweep is one launch over all of them, each scene converging on its own.
    Particles are concatenated in scene order; `first[s]` is scene s's first
    particle id and `first[-1]` the total."""

    def __init__(self, scenes):
        scenes = list(scenes)
        self.scenes = scenes
        self._cs = (PsbScene * len(scenes))(*[sc.to_c() for sc in scenes])
        h = ctypes.c_void_p()
        rc = lib().psb_create_batch(self._cs, len(scenes), ctypes.byref(h))
        if rc != OK:
            raise PsbError(rc, f"psb_create_batch: {lib().psb_status_string(rc).decode()}")
        self._h = h
        self.n = 0
        self.first = self.layout()
        self.scene = scenes[0].replace(n=int(self.first[-1]))

    def layout(self) -> np.ndarray:
        ns = ctypes.c_int32()
        self._check(lib().psb_batch_layout(self._h, ctypes.byref(ns), None), "psb_batch_layout")
        first = np.empty(ns.value + 1, np.int64)
        self._check(lib().psb_batch_layout(self._h, ctypes.byref(ns), _ptr(first)), "psb_batch_layout")
        return first

    def batch_stats(self) -> dict:
        """Per-scene arrays: iters, converged, err_final (last step), iters_total and
        unconverged_steps (since the last upload)."""
        S = len(self.scenes)
        it, cv = np.empty(S, np.int32), np.empty(S, np.int32)
        err, tot, unc = np.empty(S, np.float64), np.empty(S, np.int64), np.empty(S, np.int64)
        self._check(lib().psb_batch_stats(self._h, _ptr(it), _ptr(cv), _ptr(err), _ptr(tot), _ptr(unc)),
                    "psb_batch_stats")
        return {"iters": it, "converged": cv, "err_final": err, "iters_total": tot, "unconverged_steps": unc}

    def split(self, a: np.ndarray):
        """Per-scene views of an array in particle-id order."""
        return [a[self.first[s]:self.first[s + 1]] for s in range(len(self.scenes))]


def batch_positions(scenes) -> np.ndarray:
    return np.concatenate([scene_positions(sc) for sc in scenes])


class FluidDemCoupling:
    """Two-way coupling of a config-profile SPH context and a DEM context
    (config C1): every DEM sphere is one boundary particle of the fluid, at
    its centre.

    implicit (default): the spheres' motion is solved inside the fluid's
    pressure corrector. The spheres' gravity and contact forces at the start
    (psb_dem_forces) and their velocities go to the fluid
    (psb_set_boundary_motion); every prediction of the fluid step then also
    predicts the spheres with the fluid's reaction at that prediction's
    pressures, so the pressures and the spheres' motion converge together.
    The reaction of the last prediction is the spheres' external force in
    their own step, which moves them to that prediction.

    implicit=False: the staggered exchange -- the fluid steps with the
    spheres held, then the spheres step with its reaction. Unstable once a
    cloud of spheres as heavy as the fluid it displaces moves into the fluid
    (the added-mass effect of explicit partitioned coupling).

    Sphere positions, velocities and forces cross the host each step (12 B
    per sphere for each)."""

    def __init__(self, fluid: Simulation, spheres: Simulation, implicit: bool = True):
        self.fluid = fluid
        self.spheres = spheres
        self.implicit = implicit
        self.mass = float(spheres.scene.mass)
        self.last_force = None

    def step(self, nsteps: int = 1) -> int:
        rc = OK
        for _ in range(nsteps):
            self.fluid.set_boundary(self.spheres.read_field(FIELD_POS))
            if self.implicit:
                self.fluid.set_boundary_motion(self.spheres.read_field(FIELD_VEL), self.spheres.dem_forces(),
                                               self.mass)
            rc = max(rc, self.fluid.step(1))
            self.last_force = self.fluid.boundary_forces()
            self.spheres.set_external_force(self.last_force)
            self.spheres.step(1)
        return rc
