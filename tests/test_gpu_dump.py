"""Field dumps (SimulationData::dumpAll, SimulationData.cpp:207-239) on
the schedule of -fdump (Simulation.cpp:229, 282-297): the IC dump, then a
dump after every step that starts on a multiple of fdump.  Each field is a
float32 array with an XDMF description; its values are the fields rounded
to single precision, as the reference's DumpHDF5<..., float> writes them."""
import os
import xml.etree.ElementTree as ET

import numpy as np
import pytest

from cubismup_2d_b200 import Simulation

pytestmark = pytest.mark.gpu

ARGS = ("-bpdx 4 -bpdy 2 -extent 1 -CFL 0.1 -nu 1e-3 -poissonType freespace -muteAll 1 -fdump 2 "
        "-serialization {} -shapes 'disk radius=0.1 xpos=0.3 ypos=0.25 bForced=1 bFixed=1 xvel=0.2'")


def _read(path, ny, nx, ch):
    return np.fromfile(path, dtype="<f4").reshape(ny, nx, ch)


def test_dumps_follow_the_reference_schedule_and_fields(tmp_path):
    s = Simulation(ARGS.format(tmp_path))
    s.init()
    for _ in range(3):
        s.advance(s.calcMaxTimestep())
    names = sorted(os.listdir(tmp_path))
    for stem in ("velChi_IC0000000", "velChi_avemaria_0000001", "velChi_avemaria_0000003",
                 "pres_avemaria_0000003", "invRho_avemaria_0000003"):
        assert stem + ".raw" in names and stem + ".xmf" in names, (stem, names)
    assert not any("0000002" in n for n in names)
    ny, nx = s.ctx.ny, s.ctx.nx
    vc = _read(tmp_path / "velChi_avemaria_0000003.raw", ny, nx, 3)
    for k, f in enumerate(("u", "v", "chi")):
        assert np.array_equal(vc[:, :, k], s.ctx.get(f).astype(np.float32)), f
    p = _read(tmp_path / "pres_avemaria_0000003.raw", ny, nx, 1)[:, :, 0]
    assert np.array_equal(p, s.ctx.get("pres").astype(np.float32))
    assert np.all(_read(tmp_path / "invRho_avemaria_0000003.raw", ny, nx, 1) == 1)
    x = ET.parse(tmp_path / "velChi_avemaria_0000003.xmf").getroot()
    item = x.find(".//Attribute/DataItem")
    assert item.get("Dimensions") == f"{ny} {nx} 3" and item.text == "velChi_avemaria_0000003.raw"
    assert float(x.find(".//Time").get("Value")) == s.ctx.scalars()["time"]
