"""BCpotentials as FP64 FFT convolutions (PICARD_BCPOT_FFT, the default of
the CELL32 layout) against the oracle's direct sum (BCpotentials.f90:36-139).

Each face is a sum over the cell planes along its normal of 2-D
convolutions over its tangential axes with slices of the CalcDistance table,
evaluated with FP64 FFTs of power-of-two lengths >= 2n-1.  Bar: the face
potentials within 1e-12 relative L2 of the FP64 direct sum (both FP64; the
transforms round differently from the sum)."""
import numpy as np
import pytest

from oracle import oracle as O
from picard_b200 import capi
from picard_b200.simulation import Simulation
from tests.helpers import rel_l2, small_plasma

pytestmark = pytest.mark.gpu

BCPOT_FFT = 2


def _charged(dims, seed=23, ppc=2, **kw):
    nx, ny, nz = dims
    p = small_plasma(n=8, ppc=ppc, seed=seed, **kw)
    p.nx, p.ny, p.nz = nx, ny, nz
    p.xmin, p.xmax = -500.0 * nx, 500.0 * nx
    p.ymin, p.ymax = -500.0 * ny, 500.0 * ny
    p.zmin, p.zmax = -500.0 * nz, 500.0 * nz
    p.max_per_proc = nx * ny * nz * 8 + 100000
    p = O.derive(p)
    o = O.OracleState(p)
    o.calc_distance()
    o.initialize()
    o.step(1)
    o.step(2)
    o.gridify()
    o.bc_potentials()
    return p, o


@pytest.mark.parametrize("dims", [(16, 16, 16), (160, 24, 20), (40, 136, 12), (72, 66, 70), (33, 5, 1), (1, 1, 7)])
@pytest.mark.parametrize("layout", [capi.LAYOUT_F64, capi.LAYOUT_CELL32])
def test_bc_potentials_fft_vs_oracle(dims, layout):
    p, o = _charged(dims)
    g = Simulation(p, derive=False, layout=layout, solver=capi.SOLVER_SPECTRAL)
    if layout == capi.LAYOUT_CELL32:
        assert g.get_option(capi.OPT_BCPOT_TENSOR) == BCPOT_FFT  # the layout's default
    g.set_option(capi.OPT_BCPOT_TENSOR, BCPOT_FFT)
    g.calc_distance()
    g.set_field(capi.FIELD_C, o.C)
    g.bc_potentials()
    U = g.field(capi.FIELD_U)
    err = rel_l2(U, o.U)
    print(f"FFT BCpotentials {dims}: rel L2 vs FP64 direct sum = {err:.3e}")
    assert err < 1e-12
    # everything but the open faces is zero (BCpotentials.f90:36)
    inner = U[1:-1, 1:-1, 1:-1]
    assert not inner.any()
    g.close()


@pytest.mark.parametrize("flows", [(1, 0, 1), (0, 1, 0), (0, 0, 1)])
def test_bc_potentials_fft_periodic_axes(flows):
    # periodic axes: no faces there, and the image terms of the D table enter
    # the open faces' tangential sums
    xf, yf, zf = flows
    p, o = _charged((24, 20, 18), seed=7, xflow=xf, yflow=yf, zflow=zf)
    g = Simulation(p, derive=False, layout=capi.LAYOUT_CELL32, solver=capi.SOLVER_SPECTRAL)
    g.calc_distance()
    g.set_field(capi.FIELD_C, o.C)
    g.bc_potentials()
    err = rel_l2(g.field(capi.FIELD_U), o.U)
    print(f"FFT BCpotentials flows {flows}: rel L2 {err:.3e}")
    assert err < 1e-12
    g.close()


def test_bc_potentials_fft_follows_a_new_distance_table():
    # the slice transforms are recomputed when D changes (set_field D, or
    # CalcDistance again)
    p, o = _charged((20, 18, 16), seed=3)
    g = Simulation(p, derive=False, layout=capi.LAYOUT_CELL32, solver=capi.SOLVER_SPECTRAL)
    g.calc_distance()
    g.set_field(capi.FIELD_C, o.C)
    g.bc_potentials()
    U1 = g.field(capi.FIELD_U)
    g.set_field(capi.FIELD_D, 2.0 * o.D)
    g.bc_potentials()
    U2 = g.field(capi.FIELD_U)
    g.calc_distance()
    g.bc_potentials()
    U3 = g.field(capi.FIELD_U)
    assert rel_l2(U1, o.U) < 1e-12
    assert rel_l2(U2, 2.0 * o.U) < 1e-12
    np.testing.assert_array_equal(U3, U1)
    g.close()


def test_bc_potentials_method_option_is_checked():
    p, o = _charged((8, 8, 8))
    g = Simulation(p, derive=False, layout=capi.LAYOUT_F64, solver=capi.SOLVER_F64)
    assert g.get_option(capi.OPT_BCPOT_TENSOR) == 0  # direct sum: the F64 layout's default
    with pytest.raises(capi.PicardError):
        g.set_option(capi.OPT_BCPOT_TENSOR, 3)
    g.close()
