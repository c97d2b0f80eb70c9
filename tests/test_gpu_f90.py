"""The main loop of picard.f90 driven through the reference's subroutine
signatures (include/picard_f90.h) from a C program, against picard_gpu_run on
the same parameters: the same particles in the same slots and the same
fields, bit for bit (F64 layout, FP64 solver)."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

from picard_b200 import capi
from picard_b200 import params as P
from picard_b200.simulation import Simulation

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def build_driver(tmp_path) -> str:
    exe = str(tmp_path / "f90_main_loop")
    lib = os.path.join(ROOT, "picard_b200", "lib")
    subprocess.run(["gcc", "-std=c99", "-O1", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "f90_main_loop.c"), "-o", exe, "-L", lib, "-lpicard_gpu",
                    f"-Wl,-rpath,{lib}"], check=True)
    return exe


@pytest.mark.parametrize("case", ["open", "periodic_y_haser"])
def test_reference_signature_loop_equals_picard_gpu_run(tmp_path, case):
    if case == "open":
        p = P.config_plain_32(seed=3, n=10, ppc=4)
    else:
        p = P.config_plain_scale(seed=4, nx=24, ny=12, nz=10, ppc_ion=3)
        p.yflow = 0
    steps = 4
    prm = tmp_path / "params.bin"
    prm.write_bytes(bytes(p))
    out = tmp_path / "out.bin"
    exe = build_driver(tmp_path)
    r = subprocess.run([exe, str(prm), str(steps), str(out)], capture_output=True, text=True)
    print(r.stdout, r.stderr)
    assert r.returncode == 0, r.stderr

    g = Simulation(p, layout=capi.LAYOUT_F64, solver=capi.SOLVER_F64)
    g.calc_distance()
    g.particles_initialize()
    g.run(0, steps)
    q = g.p
    nodes = (q.nx + 2) * (q.ny + 2) * (q.nz + 2)
    raw = out.read_bytes()
    n = int(np.frombuffer(raw[:4], np.int32)[0])
    off = 4
    rp = np.frombuffer(raw[off:off + 64 * n], np.float64).reshape(n, 8)
    off += 64 * n
    ip = np.frombuffer(raw[off:off + 4 * n], np.int32)
    off += 4 * n
    fields = {}
    for name, count in (("U", nodes), ("E", 3 * nodes), ("N", q.species * nodes), ("C", nodes)):
        fields[name] = np.frombuffer(raw[off:off + 8 * count], np.float64)
        off += 8 * count
    status = int(np.frombuffer(raw[off:off + 4], np.int32)[0])
    assert status == capi.OK

    assert n == g.num_local
    rg, ig = g.particles()
    np.testing.assert_array_equal(ip, ig)
    np.testing.assert_array_equal(rp[:, :6], rg[:, :6])
    for name, f in (("U", capi.FIELD_U), ("E", capi.FIELD_E), ("N", capi.FIELD_N), ("C", capi.FIELD_C)):
        np.testing.assert_array_equal(fields[name], g.field(f).ravel(), err_msg=name)
    g.close()


def test_mismatched_arguments_are_recorded():
    # A call whose scalar arguments disagree with the attached context runs
    # nothing and records PICARD_ERR_BAD_ARG naming the argument.
    p = P.config_plain_32(seed=5, n=6, ppc=2)
    g = Simulation(p, layout=capi.LAYOUT_F64, solver=capi.SOLVER_F64)
    L = capi.lib()
    L.picard_f90_status_message.restype = C.c_char_p
    L.picard_f90_set_abort(0)
    assert L.picard_f90_attach(g._h) == capi.OK
    g.particles_initialize()
    n = C.c_int32(g.num_local)
    dt = C.c_double(g.p.dt)
    bad_cap = C.c_int32(g.p.max_per_proc + 1)
    rp0 = g.particles()[0]
    L.picard_f90_advance_position(None, C.byref(dt), C.byref(bad_cap), C.byref(n))
    assert L.picard_f90_status() == capi.ERR_BAD_ARG
    assert b"max_per_proc" in L.picard_f90_status_message()
    np.testing.assert_array_equal(g.particles()[0], rp0)  # nothing ran
    stale = C.c_int32(g.num_local - 1)
    cap = C.c_int32(g.p.max_per_proc)
    L.picard_f90_advance_position(None, C.byref(dt), C.byref(cap), C.byref(stale))
    assert L.picard_f90_status() == capi.ERR_BAD_ARG
    assert b"num_local" in L.picard_f90_status_message()
    L.picard_f90_advance_position(None, C.byref(dt), C.byref(cap), C.byref(n))
    assert L.picard_f90_status() == capi.OK
    assert not np.array_equal(g.particles()[0], rp0)
    L.picard_f90_detach()
    g.close()
