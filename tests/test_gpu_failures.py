"""Failure detection through the C ABI, with every failure made on the host.

The reference stops on a NaN norm as if converged, never caps its iterations, and handles an
oversized pressure with printf + exit(0) (gaus3mg.c:86-90, move3mg.c:2272, move3mg.c:2596).
The library returns an error code instead and the context stays usable.  None of these
cases faults the GPU: a NaN in an uploaded field is ordinary arithmetic, the iteration cap is
a host-side count, and the unsupported marker type is flagged by the kernel and read back.
"""
import numpy as np
import pytest

from conftest import golden
from i3elvis_b200 import abi, lib

pytestmark = pytest.mark.gpu

E_UNSUPPORTED, E_NOCONV, E_NAN, E_PRESSURE = -4, -5, -6, -7


def _ctx(name="sphere13", edit=None, **solver):
    p, mode, fx = golden(name)
    if edit:
        edit(p)
    buf = abi.ModelBuffers(p)
    g = lib.Context(buf, abi.make_params(mode, **solver), abi.make_file_params(mode.files[0]))
    return p, buf, g


@pytest.mark.parametrize("precision,krylov", [(0, 0), (1, 8)])
def test_nan_in_uploaded_density_gives_nan_error_and_context_recovers(precision, krylov):
    p, buf, g = _ctx(stokes_rtol=1e-8, stokes_maxcyc=200, precision=precision, krylov=krylov)
    good = buf.f32["ro"].copy()
    buf.f32["ro"][p.nodenum // 2] = np.nan
    g.upload(abi.SYNC_NODES)
    with pytest.raises(lib.I3gError) as e:
        g.stokes(0, 1e30)
    assert e.value.code == E_NAN, str(e.value)
    # restore the field: the same context solves again
    buf.f32["ro"][:] = good
    g.upload(abi.SYNC_NODES)
    g.stokes(0, 1e30)
    assert g.stats()["stokes_rel"] <= 1e-8


def test_iteration_cap_gives_noconv():
    p, buf, g = _ctx(stokes_rtol=1e-12, stokes_maxcyc=1)
    with pytest.raises(lib.I3gError) as e:
        g.stokes(0, 1e30)
    assert e.value.code == E_NOCONV, str(e.value)
    assert g.stats()["stokes_cycles"] == 1


def test_fluid_marker_type_gives_unsupported():
    """Types >= 50 are the reference's fluid markers (mark3mg.c:50-99), not implemented."""
    p, buf, g = _ctx()
    buf.markt[7] = 50
    g.upload(abi.SYNC_MARKERS)
    with pytest.raises(lib.I3gError) as e:
        g.move_markers(1e10)
    assert e.value.code == E_UNSUPPORTED, str(e.value)
    assert "fluid" in str(e.value)


def test_pressure_above_1e12_gives_pressure_error():
    """The reference exits when |P| > 1e12 Pa after a solve (move3mg.c:2272): a pinned pressure
    of 2e12 Pa in the pinning cell puts the whole field there."""
    def edit(p):
        p.head["pinit"] = 2e12
    p, buf, g = _ctx(edit=edit, stokes_rtol=1e-8)
    with pytest.raises(lib.I3gError) as e:
        g.stokes(0, 1e30)
    assert e.value.code == E_PRESSURE, str(e.value)
