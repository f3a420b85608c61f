"""The envelope swimmer (CUP2D_SHAPE_ENVELOPEFISH): StefanFish's curvature
model with the benchmark configurations' carangiform envelope
0.82 (s/L + 0.0025) / 1.0025 / L in place of its spline.  The reference has
no such swimmer, so there is no oracle run; what is checked is the part
it shares with StefanFish.  Both ramp their curvature up from zero over
the first period, so at t = 0 both midlines are straight and the placed
bodies are bitwise the same.  Under way, the weaker envelope bends the
body less than StefanFish's spline."""
import numpy as np
import pytest

from cubismup_2d_b200 import Simulation

pytestmark = pytest.mark.gpu

BASE = ("-bpdx 8 -bpdy 4 -extent 1 -CFL 0.1 -nu 1e-4 -poissonType freespace -muteAll 1 "
        "-shapes '{} L=0.18 T=1 xpos=0.4 ypos=0.25'")


def test_envelope_swimmer_starts_as_stefanfish_and_bends_less():
    a = Simulation(BASE.format("envelopefish")); a.init()
    b = Simulation(BASE.format("stefanfish")); b.init()
    assert np.array_equal(a.ctx.get("chi"), b.ctx.get("chi"))
    for key in ("M", "J", "com_x", "com_y"):
        assert a.ctx.shape(0)[key] == b.ctx.shape(0)[key], key
    # half a period: both bend; the envelope's amplitude is below the spline's
    for s in (a, b):
        s.ctx.set_scalars(0.5, 0.0, 0, 0.0, 0.0)
        s.ctx.advance(5)
        s.ctx.sync()
        assert np.all(np.isfinite(s.ctx.get("u")))
    ya = np.argwhere(a.ctx.get("chi") > 0.5)[:, 0]
    yb = np.argwhere(b.ctx.get("chi") > 0.5)[:, 0]
    assert np.ptp(ya) < np.ptp(yb)            # less lateral excursion
    assert not np.array_equal(a.ctx.get("chi"), b.ctx.get("chi"))
