"""zt_render_noalloc: the render entry point for callers that must not
allocate device memory while rendering (an engine or service whose own pool
takes the GPU's memory at start-up and fails or stalls on allocations made
behind its back, or a frame loop that cannot afford an allocator's
device-wide synchronisation).

It is checked through the C ABI against the existing entry point, zt_render,
on two calls in a row.  The tolerance is the one every render test here
uses: bit-identical f64 pixels.  This file is collected last so that a run
stopping at its first failure has already run every other test.
"""
import numpy as np
import pytest

import kat_scenes as K
import zigtrace_b200 as zt
from zigtrace_b200 import _native as N
from zigtrace_b200 import scenes

pytestmark = pytest.mark.gpu


def render_noalloc(scene: zt.Scene, o: zt.Options) -> np.ndarray:
    out = np.full(o.width * o.height * 3, np.nan)
    N.check(N.lib().zt_render_noalloc(scene.handle, N.ptr(o.record()), N.ptr(out), None))
    return out.reshape(-1, 3)


def test_noalloc_matches_zt_render_on_two_calls_in_a_row():
    cornell = scenes.cornell().build()
    demo = K.demo_scene().build()
    cornell.upload()
    demo.upload()
    oc = zt.Options(64, 48, 4, 16, seed=5)
    od = zt.Options(40, 24, 8, 8, seed=3)
    first = render_noalloc(cornell, oc)
    second = render_noalloc(demo, od)
    assert first.tobytes() == zt.render(cornell, oc).pixels.tobytes()
    assert second.tobytes() == zt.render(demo, od).pixels.tobytes()
    again = render_noalloc(cornell, oc)  # the shared scratch still holds the demo frame
    assert again.tobytes() == first.tobytes()


def test_noalloc_full_size_limit_and_errors():
    scene = scenes.cornell().build()
    scene.upload()
    side = 512  # ZT_NOALLOC_MAX_PIXELS = 512 * 512
    o = zt.Options(side, side, 1, 4)
    assert render_noalloc(scene, o).tobytes() == zt.render(scene, o).pixels.tobytes()
    with pytest.raises(zt.ZigtraceError) as ei:
        render_noalloc(scene, zt.Options(side + 1, side, 1, 4))
    assert ei.value.name == "InvalidArgument" and "maximum" in str(ei.value)
    with pytest.raises(zt.ZigtraceError) as ei:
        render_noalloc(scene, zt.Options(8, 8, 0, 4))
    assert ei.value.name == "InvalidOptions"
    other = K.demo_scene().build()  # built but never uploaded
    with pytest.raises(zt.ZigtraceError) as ei:
        render_noalloc(other, zt.Options(8, 8, 1, 4))
    assert "zt_scene_upload" in str(ei.value)
