"""The reference-signature layer (include/picard_f90.h) without a GPU.

Every entry point's argument list must be the reference subroutine's, name
for name and in order; the reference's lists come from the committed fixture
tests/golden/f90_signatures.json (made by make_f90_signatures.py from the
reference's Fortran headers).  Calls made with no context attached record
PICARD_ERR_BAD_ARG and touch no device.
"""
import ctypes as C
import json
import os
import re

from picard_b200 import capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

# reference subroutine -> entry point of include/picard_f90.h
ENTRY = {
    "CalcDistance": "picard_f90_calc_distance",
    "ParticlesInitialize": "picard_f90_particles_initialize",
    "BCinflow": "picard_f90_bc_inflow",
    "AdvancePosition": "picard_f90_advance_position",
    "ParticlesProduce": "picard_f90_particles_produce",
    "BCoutflow": "picard_f90_bc_outflow",
    "ParticlesTransfer": "picard_f90_particles_transfer",
    "ParticlesGridify": "picard_f90_particles_gridify",
    "ParticlesGridifyAll": "picard_f90_particles_gridify_all",
    "BCpotentials": "picard_f90_bc_potentials",
    "CalcEpotential": "picard_f90_calc_epotential",
    "CalcEfield": "picard_f90_calc_efield",
    "BCfields": "picard_f90_bc_fields",
    "AdvanceVelocity": "picard_f90_advance_velocity",
    "AdvanceVelocityExp": "picard_f90_advance_velocity_exp",
    "AdvanceVelocityImp": "picard_f90_advance_velocity_imp",
    "DumpParticles": "picard_f90_dump_particles",
    "DumpFields": "picard_f90_dump_fields",
}


def header_prototypes():
    text = open(os.path.join(ROOT, "include", "picard_f90.h")).read()
    text = re.sub(r"/\*.*?\*/", " ", text, flags=re.S)
    out = {}
    for m in re.finditer(r"PICARD_API\s+void\s+(picard_f90_\w+)\s*\((.*?)\)\s*;", text, re.S):
        params = [p.strip() for p in m.group(2).split(",")]
        out[m.group(1)] = [re.findall(r"(\w+)\s*$", p)[0] for p in params]
    return out


def test_every_reference_subroutine_has_its_argument_list():
    ref = json.load(open(os.path.join(ROOT, "tests", "golden", "f90_signatures.json")))
    protos = header_prototypes()
    assert set(ENTRY) == set(ref)
    assert set(protos) == set(ENTRY.values())
    for name, entry in ENTRY.items():
        want = [a.lower() for a in ref[name]["args"]]
        got = [a.lower() for a in protos[entry]]
        assert got == want, (name, ref[name]["source"])


def test_pointer_and_type_per_argument():
    # every argument is passed by reference (a pointer); integer arguments are
    # int32_t, logical ones picard_f90_logical, real*8 ones double
    text = open(os.path.join(ROOT, "include", "picard_f90.h")).read()
    text = re.sub(r"/\*.*?\*/", " ", text, flags=re.S)
    logical = {"xflow", "yflow", "zflow", "fluid", "gyration"}
    integer = {"nx", "ny", "nz", "nx_local", "ny_local", "nz_local", "species", "max_per_proc", "num_local", "ppc",
               "epp", "hpp", "ipp", "iprocs", "jprocs", "kprocs", "myid", "maxit", "int_particles",
               "writeparticles_iteration", "writefields_iteration"}
    for m in re.finditer(r"PICARD_API\s+void\s+(picard_f90_\w+)\s*\((.*?)\)\s*;", text, re.S):
        for p in (q.strip() for q in m.group(2).split(",")):
            typ, name = re.match(r"(.*?)(\w+)$", p).groups()
            assert "*" in typ, (m.group(1), p)
            base = typ.replace("const", "").replace("*", "").strip()
            if name.lower() in logical:
                assert base == "picard_f90_logical", (m.group(1), p)
            elif name.lower() in integer:
                assert base == "int32_t", (m.group(1), p)
            else:
                assert base == "double", (m.group(1), p)


def test_calls_without_a_context_record_bad_arg():
    L = capi.lib()
    L.picard_f90_detach()
    L.picard_f90_status()  # clear
    L.picard_f90_set_abort(0)
    dt = C.c_double(1e-6)
    n = C.c_int32(0)
    L.picard_f90_advance_position(None, C.byref(dt), C.byref(n), C.byref(n))
    assert L.picard_f90_status() == capi.ERR_BAD_ARG
    L.picard_f90_status_message.restype = C.c_char_p
    assert b"no context attached" in L.picard_f90_status_message()
    assert L.picard_f90_status() == capi.OK  # the query cleared it
