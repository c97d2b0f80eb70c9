"""The output path on the device (include/picard_io.h): the dumps of Write.f90
hold exactly the device state formatted as E10.4 (each line equals
picard_format_e of the value it stands for, in the reference's order and file
names), and picard_gpu_run_io's write-step branch (picard.f90:602-627) is the
per-subroutine sequence with AdvanceVelocityImp / dumps / GridifyAll /
AdvanceVelocityExp on the steps where the intervals fall due -- bit for bit."""
import math
import os

import numpy as np
import pytest

from picard_b200 import capi
from picard_b200.simulation import Simulation
from helpers import small_haser

pytestmark = pytest.mark.gpu

F64 = dict(layout=capi.LAYOUT_F64, solver=capi.SOLVER_F64)


def _start(p, **kw):
    g = Simulation(p, **kw)
    g.calc_distance()
    g.particles_initialize()
    return g


def _lines(path):
    with open(path) as f:
        return f.read().split("\n")[:-1]


def test_dump_fields_and_particles_are_the_device_state(tmp_path):
    g = _start(small_haser(nx=12, ny=8, nz=6, ppc=2), **F64)
    g.run(0, 2)
    g.particles_gridify_all()
    root = str(tmp_path / "save")
    assert g.dump_fields(root, 3) == 4
    assert g.dump_particles(root, 7) == 8
    p = g.p
    fields = {"UE": g.field(capi.FIELD_U)}
    E = g.field(capi.FIELD_E)
    N = g.field(capi.FIELD_N)
    F = g.field(capi.FIELD_F)
    for d, c in enumerate("xyz"):
        fields["E" + c] = E[..., d]
    for s in range(p.species):
        fields[f"N{s + 1}"] = N[..., s]
        for d, c in enumerate("XYZ"):
            fields[f"{c}{s + 1}"] = F[..., d, s]
    names = sorted(os.listdir(os.path.join(root, "fields")))
    assert names == sorted(f"{k}_00003_00000" for k in fields)
    nodes = (p.nx + 2) * (p.ny + 2) * (p.nz + 2)
    for k, arr in fields.items():
        got = _lines(os.path.join(root, "fields", f"{k}_00003_00000"))
        assert len(got) == nodes, k
        want = [capi.format_e(v) for v in arr.ravel()]  # x fastest, ghosts included
        assert got == want, k
    rp, ip = g.particles()
    got = _lines(os.path.join(root, "particles", "particles_00007_00000"))
    assert len(got) == len(ip) == g.num_local
    want = ["".join(capi.format_e(v) for v in row[:6]) + capi.format_e(float(s)) for row, s in zip(rp, ip)]
    assert got == want
    assert all(len(line) == 70 for line in got)
    g.close()


def test_run_io_is_the_write_step_sequence(tmp_path):
    p = small_haser(nx=12, ny=8, nz=6, ppc=2)
    a = _start(p, **F64)
    dt = a.p.dt
    root = str(tmp_path / "save")
    steps, fint, pint = 6, 2.0 * dt, 3.0 * dt
    sw, nf, np_ = a.run_io(0, steps, root, fields_interval=fint, particles_interval=pint)
    # the same iterations through the per-subroutine entry points
    b = _start(p, **F64)
    broot = str(tmp_path / "manual")
    t, fi, pi = 0.0, 0, 0
    for it in range(1, steps + 1):
        t = t + dt
        b.bc_inflow(it)
        b.advance_position()
        b.particles_produce(it)
        b.bc_outflow()
        b.particles_transfer()
        b.particles_gridify()
        b.bc_potentials()
        b.calc_epotential()
        b.calc_efield()
        b.bc_fields()
        wf, wp = math.fmod(t, fint) < dt, math.fmod(t, pint) < dt
        if wf or wp:
            b.advance_velocity_imp(0.5 * dt)
            if wp:
                pi = b.dump_particles(broot, pi)
            if wf:
                b.particles_gridify_all()
                fi = b.dump_fields(broot, fi)
            b.advance_velocity_exp(0.5 * dt)
        else:
            b.advance_velocity()
    assert (nf, np_) == (fi, pi) and fi >= 2 and pi >= 1
    for which in (capi.FIELD_U, capi.FIELD_E, capi.FIELD_N):
        np.testing.assert_array_equal(a.field(which), b.field(which))
    ra, ia = a.particles()
    rb, ib = b.particles()
    np.testing.assert_array_equal(ra[:, :6], rb[:, :6])
    np.testing.assert_array_equal(ia, ib)
    for sub in ("fields", "particles"):
        assert sorted(os.listdir(os.path.join(root, sub))) == sorted(os.listdir(os.path.join(broot, sub)))
        for name in os.listdir(os.path.join(root, sub)):
            assert _lines(os.path.join(root, sub, name)) == _lines(os.path.join(broot, sub, name)), name
    a.close()
    b.close()


def _fields_of(line: str, width: int = 10):
    return [line[k:k + width] for k in range(0, len(line), width)]


def _value(field: str) -> float:
    s = field.strip()
    if "E" not in s:  # three-digit exponent: the E is dropped
        k = max(s.rfind("+"), s.rfind("-"))
        s = s[:k] + "E" + s[k:]
    return float(s)


def test_dumps_equal_the_oracles_dumps(tmp_path):
    # picard_gpu_run_io (F64 layout, FP64 solver) against the oracle's loop
    # with the same write-step branch (picard.f90:602-627) and the oracle's
    # own E10.4 dumps (Write.f90:2-31, 34-523): the same files, line for
    # line.  Positions are bit-exact, so particle lines are identical but
    # for a velocity on a rounding boundary of its fourth digit.  A field
    # line may differ only by less than 1e-7 of the field's largest value
    # (a node where the field is a near cancellation prints its rounding).
    from oracle import oracle as O

    p = O.derive(small_haser(nx=12, ny=8, nz=6, ppc=2))
    dt = p.dt
    steps, fint, pint = 5, 2.0 * dt, 3.0 * dt
    g = Simulation(p, derive=False, **F64)
    g.calc_distance()
    g.particles_initialize()
    root = str(tmp_path / "gpu")
    g.run_io(0, steps, root, fields_interval=fint, particles_interval=pint)
    o = O.OracleState(p)
    o.calc_distance()
    o.initialize()
    oroot = str(tmp_path / "oracle")
    t, fi, pi = 0.0, 0, 0
    for it in range(1, steps + 1):
        t = t + dt
        o.bc_inflow(it)
        o.advance_position()
        o.produce(it)
        o.bc_outflow()
        o.transfer()
        o.gridify()
        o.bc_potentials()
        o.calc_epotential()
        o.calc_efield()
        o.bc_fields()
        wf, wp = math.fmod(t, fint) < dt, math.fmod(t, pint) < dt
        if wf or wp:
            o.advance_velocity(mode=2, deltat=0.5 * dt)
            if wp:
                pi = O.dump_particles(*o.particles(), oroot, pi)
            if wf:
                o.gridify_all()
                fi = O.dump_fields(o, oroot, fi)
            o.advance_velocity(mode=1, deltat=0.5 * dt)
        else:
            o.advance_velocity()
    assert fi >= 2 and pi >= 1
    compared = 0
    for sub in ("fields", "particles"):
        names = sorted(os.listdir(os.path.join(oroot, sub)))
        assert sorted(os.listdir(os.path.join(root, sub))) == names
        for name in names:
            got = _lines(os.path.join(root, sub, name))
            want = _lines(os.path.join(oroot, sub, name))
            assert len(got) == len(want), name
            differ = [(a, b) for a, b in zip(got, want) if a != b]
            if sub == "particles":
                # positions bit-exact; a velocity may sit on a rounding
                # boundary of its fourth digit: one line, one unit
                assert len(differ) <= 1, (name, differ[:3])
                for a, b in differ:
                    for fa, fb in zip(_fields_of(a), _fields_of(b)):
                        if fa != fb:
                            va, vb = _value(fa), _value(fb)
                            unit = 10.0 ** (math.floor(math.log10(max(abs(vb), 1e-300))) - 3)
                            assert abs(va - vb) <= 1.01 * unit, (name, fa, fb)
            else:
                # the FP64 field agrees with the oracle's to 1e-10 (U) and
                # 1e-7 (E, a difference of nearly equal potentials) of the
                # field's scale, so the printed values may differ only where
                # four digits resolve less than that
                scale = max(abs(_value(v)) for v in want)
                for a, b in differ:
                    assert abs(_value(a) - _value(b)) <= 1e-7 * scale, (name, a, b, scale)
                assert len(differ) <= max(2, len(want) // 100), (name, len(differ))
            compared += len(got)
    assert compared > 1000
    g.close()
