"""The C-ABI library: builds for sm_100a, loads, exports every declared symbol,
and its structs have the documented layouts.  No GPU work is launched here."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

from nexus_b200 import build, mpm
from nexus_b200.particles import COLLIDER_DTYPE, PARTICLE_DTYPE

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "nexus_mpm.h")


def declared_functions():
    text = open(HEADER).read()
    return re.findall(r"^NXM_API [\w\s\*]+?\b(nxm_\w+)\(", text, flags=re.M)


def test_library_builds_and_exports_every_declared_symbol():
    lib_path = build.build()
    names = declared_functions()
    assert len(names) >= 30
    lib = C.CDLL(lib_path)
    for n in names:
        assert hasattr(lib, n), f"{n} declared in nexus_mpm.h but not exported"
    out = subprocess.run(["nm", "-D", "--defined-only", lib_path], capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r" T (nxm_\w+)", out))
    assert exported == set(names), f"exported but undeclared: {exported - set(names)}"
    # the Python binding types every declared function
    assert set(mpm.SIGNATURES) == set(names)


def test_build_targets_sm100a_only():
    # every translation unit is compiled for sm_100a and nothing else
    assert build.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]


def test_struct_layouts_match_bindings(tmp_path):
    src = tmp_path / "layout.c"
    src.write_text(f"""
#include <stddef.h>
#include <stdio.h>
#include "{HEADER}"
int main(void) {{
  printf("%zu %zu %zu %zu %zu %zu %zu\\n", sizeof(nxm_collider), sizeof(nxm_particle_model),
         sizeof(nxm_particle), sizeof(nxm_particles_soa), sizeof(nxm_simulation_params),
         sizeof(nxm_capacities), sizeof(nxm_timestamps));
  printf("%zu %zu %zu %zu\\n", offsetof(nxm_collider, rotation), offsetof(nxm_collider, translation),
         offsetof(nxm_collider, bc_type), offsetof(nxm_collider, tri_count));
  return 0;
}}
""")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-o", str(exe), str(src)], check=True)
    a, b = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")[:2]
    sizes = list(map(int, a.split()))
    offs = list(map(int, b.split()))
    assert sizes[0] == COLLIDER_DTYPE.itemsize == 128
    assert sizes[1] == 100  # GpuParticleModel stride (models/default.rs:18)
    assert sizes[2] == PARTICLE_DTYPE.itemsize
    assert sizes[3] == C.sizeof(mpm.ParticlesSoAC)
    assert sizes[4] == C.sizeof(mpm.SimulationParamsC) == 16
    assert sizes[5] == C.sizeof(mpm.CapacitiesC)
    assert sizes[6] == C.sizeof(mpm.TimestampsC)
    assert offs == [COLLIDER_DTYPE.fields[k][1] for k in ("rotation", "translation", "bc_type", "tri_count")]


def test_no_device_is_an_error_not_a_fallback():
    """Without an sm_100 GPU the library refuses to run (there is no CPU path)."""
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if has_gpu:
        pytest.skip("a GPU is present")
    lib = mpm.load(build.build())
    h = C.c_void_p()
    assert lib.nxm_pipeline_create(C.byref(h)) == mpm.NXM_E_NO_DEVICE
    st = C.c_void_p()
    assert lib.nxm_state_create(None, C.byref(st)) == mpm.NXM_E_NO_DEVICE
    with pytest.raises(mpm.NexusError):
        mpm.MpmPipeline()
