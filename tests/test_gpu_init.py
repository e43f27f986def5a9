"""Initial conditions on the GPU: markers and bodies against the CPU restatement of in3mg.c's
generator, and the device-side initial-condition passes against the reference's."""
import numpy as np
import pytest

import init_ref
from i3elvis_b200 import abi, config, lib, model

pytestmark = pytest.mark.gpu


def _bodies():
    return [abi.box_body(3, (0.2, 0.1, 0.3), (0.7, 0.45, 0.8), ex=0.5, e=0.25),
            abi.sphere_body(4, (0.5, 0.6, 0.5), (0.25, 0.25, 0.25), 0.0, 1.0),
            abi.sphere_body(5, (0.3, 0.5, 0.6), (0.1, 0.2, 0.1), 0.5, 1.0, cylinder=True)]


def _as_dict(b):
    return {"rock": b.rock, "shape": b.shape, "x": list(b.x), "y": list(b.y), "z": list(b.z), "ex": b.ex, "e": b.e}


@pytest.mark.parametrize("shape,mnum", [((17, 13, 21), (2, 3, 2)), ((33, 33, 33), (3, 3, 3))])
def test_init_markers_match_restatement(shape, mnum):
    size = (150e3, 100e3, 200e3)
    spec = model.ModelSpec(shape=shape, size=size, mnum=mnum, multinum=1)
    xyz = model.build_markers(spec, 0)
    rocks = {2: model.Rock(), 3: model.Rock(nu=1e22), 4: model.Rock(ro=3400.0), 5: model.Rock(nu=1e20)}
    prn = model.make_prn(spec, rocks, np.full(xyz[0].size, 2, np.int8), xyz)
    buf = abi.ModelBuffers(prn)
    g = lib.Context(buf, abi.make_params(config.Mode(multinum=1, multinnn=((8, 0), (8, 16)))))
    init = abi.Init(nonstab=100, xnonstab=0.5, ynonstab=0.4, znonstab=0.3, seed=12345, background=2,
                    t_top=273.0, t_bottom=1573.0)
    bodies = _bodies()
    g.init_markers(init, bodies)
    g.download(abi.SYNC_MARKERS)
    ref = init_ref.markers(shape, size, mnum, 100, (0.5, 0.4, 0.3), 12345, 2, [_as_dict(b) for b in bodies], 273.0, 1573.0)
    for f, bf in (("x", "markx"), ("y", "marky"), ("z", "markz"), ("ex", "markex"), ("e", "marke"), ("k", "markk")):
        np.testing.assert_array_equal(buf.f32[bf], ref[f], err_msg=f)
    np.testing.assert_array_equal(buf.markt, ref["t"])
    assert set(np.unique(buf.markt)) == {2, 3, 4, 5}
    # the jitter stays within half a marker spacing of the sub-grid position
    d = size[0] / (shape[0] - 1) / mnum[0]
    assert np.all(np.abs(buf.f32["markx"] - ref["x"]) <= 0.5 * d)


def test_init_rejects_fluid_rock_types():
    spec = model.ModelSpec(shape=(9, 9, 9), size=(1e5, 1e5, 1e5), mnum=(1, 1, 1), multinum=1)
    xyz = model.build_markers(spec, 0)
    prn = model.make_prn(spec, {2: model.Rock()}, np.full(xyz[0].size, 2, np.int8), xyz)
    g = lib.Context(abi.ModelBuffers(prn), abi.make_params(config.Mode(multinum=1, multinnn=((8, 0), (8, 16)))))
    with pytest.raises(lib.I3gError) as e:
        g.init_markers(abi.Init(background=2), [abi.box_body(50, (0, 0, 0), (1, 1, 1))])
    assert e.value.code == -4
