"""CPU tests of the drop-in boundary: the C-ABI library loads, exports every
entry point include/nova_gpu.h declares, its structs have the layout the
ctypes binding assumes, and without a GPU it fails loudly (no CPU fallback)."""
import ctypes as C
import os
import re
import subprocess

import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "nova_gpu.h")


def declared_symbols():
    src = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:nova_status|const char \*)\s*(nova_\w+)\s*\(", src, re.M)))


@pytest.fixture(scope="module")
def lib():
    from novaclone_b200 import nova
    if not os.path.exists(nova.LIB_PATH):
        from novaclone_b200 import build
        build.build()
    return nova.load_library()


def test_header_declares_the_binding_list():
    from novaclone_b200.nova import EXPORTS
    assert declared_symbols() == sorted(EXPORTS)


def test_library_exports_every_declared_symbol(lib):
    out = subprocess.run(["nm", "-D", "--defined-only", lib._name], capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r"\bT (nova_\w+)", out))
    missing = [s for s in declared_symbols() if s not in exported]
    assert not missing, missing


def test_struct_layout_matches_header(tmp_path):
    from novaclone_b200 import nova
    prog = tmp_path / "layout.c"
    prog.write_text(r'''
#include <stdio.h>
#include <stddef.h>
#include "nova_gpu.h"
int main(void) {
  printf("%zu %zu %zu %zu %zu\n", sizeof(nova_mesh_desc), offsetof(nova_mesh_desc, m), offsetof(nova_mesh_desc, s2), offsetof(nova_mesh_desc, walls), sizeof(nova_bc));
  printf("%zu %zu %zu %zu %zu\n", sizeof(nova_run_desc), offsetof(nova_run_desc, dt), offsetof(nova_run_desc, t0), offsetof(nova_run_desc, poisson), sizeof(nova_state));
  return 0; }
''')
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I" + os.path.join(ROOT, "include"), str(prog), "-o", str(exe)], check=True)
    got = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()
    want = [C.sizeof(nova.MeshDesc), nova.MeshDesc.m.offset, nova.MeshDesc.s2.offset, nova.MeshDesc.walls.offset,
            C.sizeof(nova.BCDesc),
            C.sizeof(nova.RunDesc), nova.RunDesc.dt.offset, nova.RunDesc.t0.offset, nova.RunDesc.poisson.offset,
            C.sizeof(nova.State)]
    assert [int(v) for v in got] == want


@pytest.mark.parametrize("prog", ["tg_driver.cpp", "im_driver.cpp", "ops2_driver.cpp"])
def test_cpp_adapter_compiles(prog):
    """The header-only C++ adapter (include/nova/nova.hpp) builds against the C ABI."""
    src = os.path.join(ROOT, "tests", "cpp", prog)
    subprocess.run(["g++", "-std=c++17", "-Wall", "-Werror", "-fsyntax-only", "-I" + os.path.join(ROOT, "include"),
                    src], check=True)


def test_invalid_arguments_rejected_without_gpu(lib):
    from novaclone_b200 import nova
    h = C.c_void_p()
    d = nova.MeshDesc()
    d.N[:] = [8, 8, 8]
    d.L[:] = [1.0, 1.0, 1.0]
    d.m = 5  # not an even order
    assert lib.nova_create(C.byref(d), C.byref(h)) == nova.E_INVALID
    assert lib.nova_advance(None, None, None, 1, None) == nova.E_INVALID


def test_implicit_operators_reject_null_handles(lib):
    """Every nova_fdm_* entry point (and nova_im_laplacian) refuses a missing
    context, matrix or field with NOVA_E_INVALID before touching the device."""
    from novaclone_b200 import nova
    h = C.c_void_p()
    its, res = C.c_int(), C.c_double()
    assert lib.nova_im_laplacian(None, 1.0, None, C.byref(h)) == nova.E_INVALID
    calls = [lib.nova_fdm_add(None, None, 1.0, None), lib.nova_fdm_mul(None, None, None),
             lib.nova_fdm_scale(None, None, -1.0), lib.nova_fdm_add_source(None, None, 1.0, None),
             lib.nova_fdm_add_diagonal(None, None, 1.0), lib.nova_fdm_relax(None, None, 0.5),
             lib.nova_fdm_set_reference(None, None, 0, 0, 0, 1.0), lib.nova_fdm_residual(None, None, C.byref(res)),
             lib.nova_fdm_solve(None, None, 0.0, 1, C.byref(its), C.byref(res)), lib.nova_fdm_download(None, None, None)]
    assert calls == [nova.E_INVALID] * len(calls)
    assert lib.nova_fdm_destroy(None) == nova.OK


def test_no_silent_cpu_fallback(lib):
    """On a machine without a GPU, creating a context fails with a CUDA error."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from novaclone_b200 import nova
    with pytest.raises(nova.NovaError) as e:
        nova.Mesh((8, 8, 8))
    assert e.value.status == nova.E_CUDA
