"""Checkpoint / restart through the handle (grid::dump / grid::load,
grid.cpp:367-381 and 482-499; the restart flow of timestepper.cpp:386-445
and torus/problem.cpp:880-907): a dumped state loads back bit for bit with
communicate's ghosts, and a run restarted from a dump continues exactly as
the uninterrupted run (FP64 parity path)."""
import numpy as np
import pytest

from grim_b200 import config as C
from grim_b200 import problems as PR
from grim_b200.problems import torus as T

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", ["periodic_2d", "torus_3d"])
def test_dump_load_round_trip(case, tmp_path):
    from grim_b200.timestepper import timeStepper
    if case == "periodic_2d":
        cfg = PR.fast_mode_config(N=40)
    else:
        cfg = T.torus_config(N1=24, N2=16, N3=8)
    a, b = timeStepper(cfg), timeStepper(cfg)
    P = np.random.default_rng(3).uniform(0.5, 1.5, (a.dof,) + a.zshape)
    a.primOld.setVars(P)
    f = tmp_path / "prims.bin"
    a.dump(f)
    raw = np.fromfile(f, dtype=">f8", offset=8)
    s3, s2, s1 = C.interior_slices(cfg)
    assert np.array_equal(raw, np.moveaxis(P[:, s3, s2, s1], 0, -1).ravel())
    b.load(f)
    Q = b.primOld.getVars()
    # the interior from the file; periodic ghosts wrapped, other ghosts zero
    assert np.array_equal(Q, T.communicate(cfg, P))


def test_restart_continues_the_run(tmp_path, monkeypatch):
    from grim_b200.timestepper import timeStepper
    monkeypatch.chdir(tmp_path)
    cfg = PR.fast_mode_config(N=64)
    P = PR.fast_mode_prims(cfg)
    a, b = timeStepper(cfg), timeStepper(cfg)
    for ts in (a, b):
        ts.primOld.setVars(P)
    for _ in range(4):
        a.timeStep()
    for _ in range(2):
        b.timeStep()
    name = b.writeRestart("restartFileName.txt", "restartFileTime.txt")
    assert (tmp_path / name).exists() and name.startswith("restartVarsT") and len(name) == len("restartVarsT") + 8 + 4
    assert (tmp_path / "restartFileName.txt").read_text().split()[0] == name
    t_b, dt_b = b.time, b.dt
    assert float((tmp_path / "restartFileTime.txt").read_text()) == float("%g" % t_b)
    c = timeStepper(cfg)
    c.restart("restartFileName.txt", "restartFileTime.txt")
    assert c.time == float("%g" % t_b)
    c.setTime(c.time, dt_b)  # the dt a restarted run starts from is the caller's
    for _ in range(2):
        c.timeStep()
    assert np.array_equal(c.primOld.getVars(), a.primOld.getVars())


def test_restart_without_files_is_an_error(tmp_path, monkeypatch):
    from grim_b200.timestepper import timeStepper
    from grim_b200._lib import GrimError
    monkeypatch.chdir(tmp_path)
    ts = timeStepper(PR.fast_mode_config(N=16))
    with pytest.raises(GrimError):
        ts.restart("none.txt", "none2.txt")
    with pytest.raises(GrimError):
        ts.restart("none.txt", "none2.txt", restartFile="missing.bin")
