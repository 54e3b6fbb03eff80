"""The RendererObserver contract of render(int) (renderer/gpu/AbstractGPURenderer.java:231-332):
every pass notifies onRenderPassProgress(0.0), then, after the pass and the
image update, onRenderPassProgress(1.0), onRenderDisplay(image) and
onRenderPassComplete(renderPass, millis); the first pass after a clear shows
the cleared image first."""
import numpy as np
import pytest

from dayflower_b200 import GPURenderer, RenderingAlgorithm as RA
from dayflower_b200.renderer import DFC_E_STATE, RenderError
from dayflower_b200.scene import generators as G
from dayflower_b200.scene.compiler import compile_scene

pytestmark = pytest.mark.gpu


class Recorder:
    def __init__(self):
        self.events = []
        self.last_image = None

    def onRenderPassProgress(self, renderer, render_pass, progress):
        self.events.append(("progress", render_pass, progress))

    def onRenderDisplay(self, renderer, image):
        self.events.append(("display",))
        self.last_image = image

    def onRenderPassComplete(self, renderer, render_pass, millis):
        assert millis > 0.0
        self.events.append(("complete", render_pass))


def test_observer_sees_every_pass_and_the_image():
    cs = compile_scene(G.cornell_box(resolution=(96, 64)))
    rec = Recorder()
    r = GPURenderer(renderer_observer=rec)
    try:
        r.setScene(cs)
        r.setRenderingAlgorithm(RA.PATH_TRACING)
        r.setMaximumBounce(6)
        r.setup()
        assert r.render(4)
        want = [("display",)]
        for k in range(1, 5):
            want += [("progress", k, 0.0), ("progress", k, 1.0), ("display",), ("complete", k)]
        assert rec.events == want
        assert rec.last_image.shape == (64, 96, 4)
        assert np.array_equal(rec.last_image, r.getImage())
        # render(int) continues the pass count; a clear starts it again with the cleared image
        rec.events.clear()
        assert r.render(1)
        assert rec.events == [("progress", 5, 0.0), ("progress", 5, 1.0), ("display",), ("complete", 5)]
        r.clear()
        rec.events.clear()
        assert r.render(1)
        assert rec.events[0] == ("display",) and rec.events[1] == ("progress", 1, 0.0)
        # the observed render accumulates the same film as a plain one
        s_obs, _, n_obs = r.getFilm()
    finally:
        r.dispose()
    q = GPURenderer()
    try:
        q.setScene(cs)
        q.setRenderingAlgorithm(RA.PATH_TRACING)
        q.setMaximumBounce(6)
        q.setup()
        q.render(1)
        s, _, n = q.getFilm()
    finally:
        q.dispose()
    assert np.array_equal(n, n_obs)
    assert np.allclose(s, s_obs, rtol=1e-5, atol=1e-6)


def test_observer_may_stop_but_not_reenter():
    cs = compile_scene(G.cornell_box(resolution=(32, 32)))

    class Stopper:
        def __init__(self):
            self.codes = []

        def onRenderPassComplete(self, renderer, render_pass, millis):
            try:
                renderer.getCounters()  # a call back into the rendering handle is refused
            except RenderError as e:
                self.codes.append(e.code)
            if render_pass == 2:
                renderer.renderShutdown()

    st = Stopper()
    r = GPURenderer(renderer_observer=st)
    try:
        r.setScene(cs)
        r.setup()
        assert not r.render(10)  # stopped after the second pass
        assert r.getRenderPass() == 2
        assert st.codes == [DFC_E_STATE, DFC_E_STATE]
    finally:
        r.dispose()
