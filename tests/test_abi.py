"""C ABI checks that need no GPU: the library loads, exports every entry
point include/psb.h declares, its structs have the layout the bindings use,
and the host-side scene generator matches the oracle's bit for bit."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

import oracle
import psb_project_b200 as P
from psb_project_b200 import runtime as R
from psb_project_b200.colliders import PsbCollider
from psb_project_b200.emitters import PsbEmitter
from psb_project_b200.scene import PsbScene

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "psb.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:int|int32_t|const char\*)\s+(psb_\w+)\s*\(", src, flags=re.M)))


def test_every_declared_symbol_is_exported():
    names = declared_functions()
    assert len(names) >= 15
    L = R.lib()
    for n in names:
        assert hasattr(L, n), n
    assert set(names) == set(R.EXPORTS)
    out = subprocess.run(["nm", "-D", "--defined-only", R.LIB_PATH], capture_output=True, text=True).stdout
    for n in names:
        assert re.search(rf"\bT {n}\b", out), n


def test_header_constants_match_bindings():
    src = open(HEADER).read()
    defs = dict(re.findall(r"^#define\s+(PSB_\w+)\s+(\d+)\b", src, flags=re.M))
    assert int(defs["PSB_MLP_SILU6"]) == R.MLP_SILU6 and int(defs["PSB_MLP_RELU7"]) == R.MLP_RELU7
    assert int(defs["PSB_CORRECTOR_LAUNCHES"]) == R.CORRECTOR_LAUNCHES
    assert int(defs["PSB_CORRECTOR_PERSISTENT"]) == R.CORRECTOR_PERSISTENT
    assert int(defs["PSB_MLP_PARAMS"]) == R.mlp_params(R.MLP_RELU7)
    assert int(defs["PSB_MLP_PARAMS_SILU6"]) == R.mlp_params(R.MLP_SILU6)


def test_struct_layout_matches_header(tmp_path):
    c = tmp_path / "layout.c"
    c.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "psb.h"\n'
                 'int main(void){printf("%zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu\\n", sizeof(psb_scene), offsetof(psb_scene, spacing),'
                 ' sizeof(psb_step_stats), offsetof(psb_step_stats, iters_total), offsetof(psb_scene, dem_attraction),'
                 ' sizeof(psb_iso_grid), offsetof(psb_iso_grid, scale), sizeof(psb_tune), offsetof(psb_tune, ms),'
                 ' sizeof(psb_diag), offsetof(psb_diag, density_err_max));'
                 ' printf("%zu %zu %zu %zu %zu %zu\\n", sizeof(psb_collider), offsetof(psb_collider, v),'
                 ' offsetof(psb_collider, data), sizeof(psb_emitter), offsetof(psb_emitter, data),'
                 ' offsetof(psb_emitter, seed));'
                 ' return 0;}\n')
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(c), "-o", str(exe)], check=True)
    got = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True).stdout.split()]
    assert got == [ctypes.sizeof(PsbScene), PsbScene.spacing.offset, ctypes.sizeof(R.PsbStepStats),
                   R.PsbStepStats.iters_total.offset, PsbScene.dem_attraction.offset, ctypes.sizeof(R.IsoGrid),
                   R.IsoGrid.scale.offset, ctypes.sizeof(R.PsbTune), R.PsbTune.ms.offset,
                   ctypes.sizeof(R.PsbDiag), R.PsbDiag.density_err_max.offset,
                   ctypes.sizeof(PsbCollider), PsbCollider.v.offset, PsbCollider.data.offset,
                   ctypes.sizeof(PsbEmitter), PsbEmitter.data.offset, PsbEmitter.seed.offset]


def test_abi_version_and_status_strings():
    L = R.lib()
    assert L.psb_abi_version() == 2
    assert L.psb_status_string(0) == b"ok"
    assert L.psb_status_string(3) == b"neighbour list overflow"
    assert L.psb_status_string(99) == b"unknown status"


@pytest.mark.parametrize("name", ["C0", "C1", "C2"])
def test_scene_generator_matches_oracle_bitwise(name):
    sc = P.config_scene(name)
    a = P.scene_positions(sc)
    b = oracle.scene_positions(sc)
    assert a.shape == (sc.n, 3)
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    # inside the box, jitter within bounds
    blk = sc.blocks[0]
    ideal = np.stack(np.meshgrid(*[np.arange(k) for k in blk.nxyz], indexing="ij"), -1)
    ideal = (ideal.transpose(2, 1, 0, 3).reshape(-1, 3) + 0.5) * blk.spacing
    assert np.max(np.abs(a - ideal)) <= blk.jitter + float(np.spacing(np.float32(ideal.max())))


def test_lattice_rejects_bad_arguments():
    L = R.lib()
    out = np.empty((8, 3), np.float32)
    nx = np.array([2, 2, 0], np.int32)
    org = np.zeros(3)
    assert L.psb_lattice(nx.ctypes.data_as(ctypes.c_void_p), 0.01, org.ctypes.data_as(ctypes.c_void_p), 0.0, 0, 0,
                         out.ctypes.data_as(ctypes.c_void_p)) == R.EINVAL


def test_create_rejects_invalid_scene():
    sc = P.config_scene("C0").replace(max_iters=1000)
    with pytest.raises(R.PsbError) as e:
        P.Simulation(sc)
    assert e.value.status == R.EINVAL


def test_library_fails_loudly_when_missing(monkeypatch):
    monkeypatch.setattr(R, "_lib", None)
    monkeypatch.setattr(R, "LIB_PATH", "/nonexistent/libpsb.so")
    with pytest.raises(ImportError):
        R.lib()


def test_every_compat_launcher_is_exported():
    """include/psb_compat.h: the reference's launchers under their own names."""
    src = open(os.path.join(ROOT, "include", "psb_compat.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = sorted(set(re.findall(r"^\s*void\s+(\w+)\s*\(", src, flags=re.M)))
    assert {"createGrid", "storeParticles", "searchNeighbooring", "pci_SPH_update", "interactionSystem",
            "collisionSystem_Box_CUDA"} <= set(names)
    out = subprocess.run(["nm", "-D", "--defined-only", R.LIB_PATH], capture_output=True, text=True).stdout
    for n in names:
        assert re.search(rf"\bT {n}\b", out), n


@pytest.mark.parametrize("header", ["psb.h", "psb_compat.h"])
@pytest.mark.parametrize("lang", [("gcc", "-std=c99", "c"), ("g++", "-std=c++17", "cpp")])
def test_header_compiles_strictly(tmp_path, header, lang):
    """The public headers build warning-free as C99 and C++17 under -pedantic,
    as a C or C++ host would include them."""
    cc, std, ext = lang
    src = tmp_path / f"inc.{ext}"
    src.write_text(f'#include "{header}"\n')
    cuda_inc = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "include")
    r = subprocess.run([cc, std, "-Wall", "-Wextra", "-pedantic", "-Werror", "-fsyntax-only",
                        "-I", os.path.join(ROOT, "include"), "-I", cuda_inc, str(src)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
