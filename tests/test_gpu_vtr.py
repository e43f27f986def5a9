"""ParaView output from device memory: the file's coordinates and nodal fields equal the
context's arrays (reordered from VTK's x-fastest point order)."""
import numpy as np
import pytest

from conftest import golden
from i3elvis_b200 import abi, lib, runtime
from i3elvis_b200.vtr import read_vtr, to_model_order

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["sphere13", "stretch17"])
def test_vtr_matches_device_fields(name, tmp_path):
    p, mode, fx = golden(name)
    buf = abi.ModelBuffers(p)
    g = lib.Context(buf, abi.make_params(mode, stokes_rtol=1e-8), abi.make_file_params(mode.files[0]))
    runtime.time_step(g, mode, mode.files[0], 0)
    g.download(abi.SYNC_ALL)
    path = str(tmp_path / "out.vtr")
    g.write_vtr(path)
    v = read_vtr(path)
    assert v["extent"] == tuple(p.shape)
    for a, gl in (("xcoor", buf.gx), ("ycoor", buf.gy), ("zcoor", buf.gz)):
        np.testing.assert_array_equal(v[a], gl.astype(np.float64))
    for f, src in (("viscosity", buf.f32["nu"]), ("temperature", buf.f32["tk"]), ("density", buf.f32["ro"]),
                   ("vx", buf.f32["vx"]), ("vy", buf.f32["vy"]), ("vz", buf.f32["vz"]), ("pressure", buf.pr)):
        assert v[f].dtype == src.dtype, f
        np.testing.assert_array_equal(to_model_order(v[f], v["extent"]), src, err_msg=f)
