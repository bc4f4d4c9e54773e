"""Batches over several scenes (the batched-jobs workload: receiver/occluder
pairs of different sizes, resolutions and light scales in one engine run)."""
import numpy as np
import pytest

from conftest import scene

pytestmark = pytest.mark.gpu


def _jobs():
    from beamtrace2007_b200 import scenes
    from beamtrace2007_b200.renderer import PreparedScene
    out = []
    for seed, tris, res, scale in ((3, 2000, 64, 0.5), (4, 12000, 128, 2.0), (5, 30000, 96, 1.0)):
        s = scenes.shadow_job(seed, tris)
        out.append((s, PreparedScene(s.pos, s.tris), res, scale))
    return out


def test_multi_scene_batch_equals_jobs_alone(gpu):
    """One context holding four scenes; a batch mixing them gives each job
    bitwise what a context holding only its scene gives alone."""
    from beamtrace2007_b200.renderer import GpuRenderer, make_camera
    s0, ps0 = scene("plant")
    jobs = _jobs()
    with GpuRenderer(ps0) as g:
        ids = [0] + [g.add_scene(ps) for _, ps, _, _ in jobs]
        assert ids == [0, 1, 2, 3]
        v0 = s0.views[0]
        cams = [make_camera(v0.eye, v0.target, v0.fov, s0.up, 80, 60)]
        lights = [s0.light_array(1.0)]
        for s, ps, res, scale in jobs:
            v = s.views[0]
            cams.append(make_camera(v.eye, v.target, v.fov, s.up, res, res))
            lights.append(s.light_array(scale))
        order = [3, 0, 1, 2, 0]  # scene of each job (scene 0 twice)
        batch = g.batch_soft([cams[k] for k in order], [lights[k] for k in order], exact=True, scenes=order)
    alone = {}
    for k, (sd, ps) in enumerate([(s0, ps0)] + [(s, ps) for s, ps, _, _ in jobs]):
        with GpuRenderer(ps) as r:
            alone[k] = r.soft_shadows(cams[k], lights[k], exact=True)
    for k, b in zip(order, batch):
        for f in ("tri", "vis", "E", "Eu"):
            assert np.array_equal(getattr(b, f), getattr(alone[k], f)), (k, f)
    # the first job's own scene after three others were added
    assert batch[1].vis.size == 80 * 60 and (batch[1].tri >= 0).any()
