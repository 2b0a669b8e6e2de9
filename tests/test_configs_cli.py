"""The benchmark-configuration runner's command line and parameters (host
only: the runs themselves are replaced by recorders, no device is used).

`python -m lbx.configs cfg3` runs the 192 x 192 x 384 flow + solute case;
`--edge E` scales it to E x E x 2E and `--quick` keeps only the FP32 run
between the faces (for short runs under a profiler).
"""
import json

import pytest

from lbx import configs


@pytest.fixture
def recorded(monkeypatch, capsys):
    calls = []

    def fake_run_cfg3(steps=20000, shape=(192, 192, 384), chunk=1000, quick=False):
        calls.append(dict(steps=steps, shape=tuple(shape), quick=quick))
        return [{"config": "cfg3", "steps": steps}]
    monkeypatch.setattr(configs, "run_cfg3", fake_run_cfg3)
    return calls, capsys


@pytest.mark.parametrize("argv,want", [
    (["cfg3"], dict(steps=20000, shape=(192, 192, 384), quick=False)),
    (["cfg3", "--steps", "200", "--quick"], dict(steps=200, shape=(192, 192, 384), quick=True)),
    (["cfg3", "--steps", "40", "--edge", "128", "--quick"],
     dict(steps=40, shape=(128, 128, 256), quick=True)),
])
def test_cfg3_command_line(recorded, argv, want):
    calls, capsys = recorded
    assert configs.main(argv) == 0
    assert calls == [want]
    line = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    assert line["config"] == "cfg3" and line["steps"] == want["steps"]


def test_cfg3_params_faces_and_planes():
    """With faces: Zou-He density on the bottom and top planes, C = 1 held
    at the bottom, zero gradient on top, both face planes kept fluid; the
    closed box has none of them."""
    p, mask = configs.cfg3_params(4, (16, 12, 24))
    assert (p.LX, p.LY, p.LZ, p.nsubs, p.precision) == (16, 12, 24, 2, 4)
    m3 = mask.reshape(24, 12, 16)
    assert not m3[0].any() and not m3[-1].any()
    assert tuple(p.pressure_b_in) == (1, 0) and tuple(p.pressure_t_out) == (1, 0)
    assert p.constcon_b_in == 1 and p.zeroconcgrad_t == 1
    p2, _ = configs.cfg3_params(8, (16, 12, 24), faces=False)
    assert p2.precision == 8
    assert tuple(p2.pressure_b_in) == (0, 0) and p2.constcon_b_in == 0 and p2.zeroconcgrad_t == 0
