"""The walk's cycle guard on the oracle: a ray that comes back to a cell with
no hit since ends there (the reference's loop would never return); a cycle
that absorbs keeps walking until the transmittance ends it; the step cap
still comes first."""

import numpy as np

from oracle import oracle as orc
from tests.helpers import cycle_scene, orc_cam, packed


def _trace(cycle_density, **kw):
    sc, adj, off, faces, cam = cycle_scene(cycle_density)
    sph, nsig, _ = packed(sc)
    return orc.trace_forward(orc_cam(cam), sph, nsig, sc["texel_sites"], sc["texel_rgb"], sc["texel_height"], adj,
                             off, faces.view(np.uint16), 0, visit_cap=16, **kw)


def test_cycle_without_hits_ends_the_walk():
    o = _trace(0.0)
    assert (o["status"] == 0).all()
    # saves at steps 0, 1, 2: cell 2 saved at step 2 comes back at step 4
    assert (o["visit_count"] == 4).all()
    assert (o["visits"][..., :4] == np.array([0, 1, 2, 1])).all()
    assert (o["color"].sum(-1) > 0).all()  # cell 0's segment is composited
    base = _trace(0.0, thr=0.999)  # cell 0 alone takes the transmittance below 0.999
    assert (base["visit_count"] == 1).all()


def test_cycle_with_hits_walks_on_to_the_threshold():
    o = _trace(3.0)
    assert (o["status"] == 0).all()
    assert (o["visit_count"] > 4).all()
    assert (np.exp(o["log_t"]) < 1e-3).all()


def test_step_cap_comes_before_the_guard():
    o = _trace(0.0, max_steps=3)
    assert (o["status"] == 2).all() and (o["visit_count"] == 3).all()
