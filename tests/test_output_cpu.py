"""The output path on the host (include/picard_io.h) without a GPU: the
Fortran E edit descriptor of Write.f90 / WriteWarnings.f90, the plasma
quantities and warnings of WriteWarnings.f90 against a restatement here, and
the parameters.dat / warnings.dat files read back the way the reference's plot
scripts read them (loadPar: split at '=', first float or T/F)."""
import math
import os

import numpy as np
import pytest

from picard_b200 import capi
from picard_b200 import params as P

# Fortran 2008 10.7.2.3.3 (E editing, scale factor 0): 0.d..d E+ee, the optional
# leading zero dropped when the sign needs its column, E omitted for 3-digit
# exponents; gfortran's words for NaN and Infinity.
E10_4 = [
    (1.0, "0.1000E+01"), (-1.0, "-.1000E+01"), (0.0, "0.0000E+00"), (12345.678, "0.1235E+05"),
    (-0.000123456, "-.1235E-03"), (9.99996, "0.1000E+02"), (0.00001, "0.1000E-04"), (1e-100, "0.1000E-99"),
    (1e-101, "0.1000-100"), (1.5e200, "0.1500+201"), (-2.5e-250, "-.2500-249"), (0.5, "0.5000E+00"),
    (float("nan"), "       NaN"), (float("inf"), "  Infinity"), (float("-inf"), " -Infinity"),
]


@pytest.mark.parametrize("value,text", E10_4)
def test_e10_4(value, text):
    assert capi.format_e(value, 10, 4) == text


def test_e12_6_and_overflow():
    assert capi.format_e(6.0221e23, 12, 6) == "0.602210E+24"
    assert capi.format_e(-1.60217646e-19, 12, 6) == "-.160218E-18"
    assert capi.format_e(1e-320, 12, 6) == "0.999989-320"
    assert capi.format_e(-1.0, 6, 4) == "******"  # -.1000E+01 needs 10 columns


def _plasma_restated(p):
    """WriteWarnings.f90:40-115 and 261-496 restated with numpy (maxval over
    species 2..8 ignores NaN, as gfortran's MAXVAL does)."""
    tau, ec, me, c0 = 6.2831853071795864769252867665590, 1.60217646e-19, 9.1093819e-31, 2.99792458e8
    mu0, eps0, kb = 1.25663706143591729538505735331180e-6, 8.854187817e-12, 1.380650e-23
    mass, charge, dens, kel = (np.array(getattr(p, k)[:8], float) for k in ("mass", "charge", "density", "kelvin"))
    v04 = [p.v0[s][3] for s in range(8)]
    B4 = p.B0[3]
    with np.errstate(all="ignore"):
        vth = np.sqrt(2.0 * kb * kel / (mass + 1e-99))
        freq = 1.0 / p.dt
        wp = [math.sqrt(dens[0] * charge[0] ** 2 / mass[0] / eps0),
              np.nanmax(np.sqrt(dens[1:] * charge[1:] ** 2 / mass[1:] / eps0)),
              math.sqrt(dens[0] * ec ** 2 / me / eps0)]
        wc = [abs(charge[0]) * B4 / mass[0], np.nanmax(np.abs(charge[1:]) * B4 / mass[1:]), ec * B4 / me]
        va = B4 / math.sqrt(mu0 * float(np.sum(mass * dens)))
        vc = [vth[0] * math.sqrt(0.5), np.nanmax(vth[1:] * math.sqrt(0.5)), vth[0] * math.sqrt(0.5 * mass[0] / me)]
        if not p.gyration[0]:
            wc[0] = wc[1]
        Ld = [vc[k] / wp[k] for k in range(3)]
        rL = [vc[k] / wc[k] for k in range(3)]
        rPU = [v04[0] / wc[k] for k in range(3)]
        Li = [va / wc[k] for k in range(3)]
        dx = p.dxyz[0]
        cfl = dx / p.dt
    conds = [wp[0] > freq, wp[1] > freq, wc[0] > freq, wc[1] > freq, va > cfl, v04[0] + vth[0] > cfl,
             v04[1] + vth[1] > cfl, Ld[0] < dx, Ld[1] < dx, rL[0] < dx, rL[1] < dx, rPU[0] < dx, rPU[1] < dx,
             Li[0] < dx, Li[1] < dx, p.dxyz[0] != p.dxyz[1] or p.dxyz[1] != p.dxyz[2],
             sum(p.Qn[s] * p.ppc[s] for s in range(8)) > 0.0]
    mask = sum(1 << k for k, c in enumerate(conds) if c)
    dt_c = 1.0 / math.sqrt(3.0) * dx / c0
    dt_part = 1.0 / math.sqrt(3.0) * dx / (max(2.0 * v04[0], 2.0 * v04[1]) + math.sqrt(12.0 / tau) * max(vc[0], vc[1]))
    dt_wave = tau / math.sqrt(12.0) / max(wc[0], wc[1], wp[0], wp[1])
    return {"wp": wp, "wc": wc, "va": va, "vc": vc, "Ld": Ld, "rL": rL, "cfl": cfl, "mask": mask,
            "dt_opt": max(min(dt_part, dt_wave), dt_c)}


@pytest.mark.parametrize("make", [lambda: P.config_plain_32(), lambda: capi.params_default(),
                                  lambda: P.config_plain_scale(nx=16, ny=8, nz=8)])
def test_plasma_quantities_and_warnings(make):
    p = capi.params_derive(make())
    got = capi.plasma(p)
    ref = _plasma_restated(p)
    for k in ("wp", "wc", "vc", "Ld", "rL"):
        np.testing.assert_allclose(got[k], ref[k], rtol=1e-14, err_msg=k)
    for k in ("va", "cfl", "dt_opt"):
        assert got[k] == pytest.approx(ref[k], rel=1e-14), k
    assert got["warnings"] == ref["mask"]


def _load_par(path, name):
    # the reference's loadPar (example_fieldplot.py:26-59)
    with open(path) as f:
        for line in f:
            if name in line:
                for tok in line.split("=")[1].split():
                    try:
                        return float(tok)
                    except ValueError:
                        if tok == "T":
                            return 1.0
                        if tok == "F":
                            return 0.0
    raise KeyError(name)


def test_parameter_and_warning_files(tmp_path):
    p = capi.params_derive(P.config_plain_scale(nx=16, ny=8, nz=8))
    root = str(tmp_path / "save")
    mask = capi.write_parameters(p, root)
    par = os.path.join(root, "parameters.dat")
    for s in range(8):
        for name, arr in (("density", p.density), ("mass", p.mass), ("n2p", p.n2p), ("Qn", p.Qn)):
            v = _load_par(par, f"{name}_{s + 1} ")
            assert v == pytest.approx(arr[s], rel=1e-6, abs=0.0), (name, s)
        assert _load_par(par, f"ppc_{s + 1} ") == p.ppc[s]
        assert _load_par(par, f"gyration_{s + 1} ") == (1.0 if p.gyration[s] else 0.0)
    assert _load_par(par, "dxyz_1") == pytest.approx(p.dxyz[0], rel=1e-6)
    assert _load_par(par, "Nx") == p.nx and _load_par(par, "xflow") == 1.0
    # every E12.6 field is 12 columns
    for line in open(par):
        if "gyration" in line or "flow" in line or "ppc" in line or "procs" in line or line.startswith("N"):
            continue
        assert len(line.rstrip("\n").split(" = ")[1]) == 12, line
    text = open(os.path.join(root, "warnings.dat")).read()
    assert mask == capi.plasma(p)["warnings"]
    for t in capi.warning_texts(mask):
        assert t in text
    assert text.count("****\n") == 2 * bin(mask).count("1")


@pytest.mark.parametrize("value,text", E10_4)
def test_oracle_e10_4(value, text):
    # the oracle's own restatement of Ew.d, which the dump parity test
    # formats the oracle's arrays with
    from oracle import oracle as O

    assert O.format_e(value, 10, 4) == text
