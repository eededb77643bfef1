"""The NetCDF writer (canoe_b200.output), the main loop (canoe_b200.driver)
and the examples' regression check, on the CPU.

- layout: the reference's dimensions, coordinate attributes and the
  (time, x1, x2, x3) transpose of every cell variable (netcdf.cpp:106-454);
- the potential temperature of the rising-bubble initial state against its
  closed form: theta = Ts on the dry adiabat, Ts + dT inside the bubble's
  core (robert.cpp:72-114);
- per-block files joined by the domain_decomposition attributes equal the
  whole-domain file (CombineBlocks / mppnccombine);
- the L2 check of test_robert.py / test_straka.py: passes on equal files,
  fails with the example's message on a planted difference above the
  threshold;
- the main loop: the last step cut to end at tlim, outputs at the start,
  when next_time is reached, and at the end;
- the committed golden of the robert2d run: its header and the physical
  bounds of theta (materially conserved in the dry adiabatic flow).
"""
import os

import numpy as np
import pytest
from scipy.io import netcdf_file

from canoe_b200 import driver, output, partition, problems
from canoe_b200._abi import NGHOST

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden",
                      "robert2d_ppm.theta.01080s.nc")


class _Block:
    """A MeshBlock-like source holding a fixed primitive state."""

    def __init__(self, problem, w):
        self.problem, self.w = problem, w

    def primitive(self):
        return self.w


class _Mesh:
    """A Mesh-like source: a split domain and its blocks' states."""

    def __init__(self, problem, nb2, nb3):
        self.split = partition.split(problem, nb2, nb3)
        c = problem.cfg
        ks = NGHOST if c.nx3 > 1 else 0
        js = NGHOST if c.nx2 > 1 else 0
        self.blocks = []
        for p, (o2, o3) in zip(self.split.blocks, self.split.offsets):
            w = np.zeros(p.u.shape)
            kb = slice(NGHOST, NGHOST + p.cfg.nx3) if p.cfg.nx3 > 1 else slice(0, 1)
            jb = slice(NGHOST, NGHOST + p.cfg.nx2) if p.cfg.nx2 > 1 else slice(0, 1)
            w[:, kb, jb, :] = problem.w[:, ks + o3:ks + o3 + p.cfg.nx3,
                                        js + o2:js + o2 + p.cfg.nx2, :]
            self.blocks.append(_Block(p, w))


def _c2():
    return problems.moist3d(nx1=12, nx2=12, nx3=6, x1max=3000.0, x2max=4000.0, x3max=3000.0,
                            noise=0.5)


def test_layout_and_transpose(tmp_path):
    p = _c2()
    o = output.NetcdfOutput(str(tmp_path / "c2"), dt=1.0)
    (path,) = o.write(_Block(p, p.w), 0.0)
    assert os.path.basename(path) == "c2.out2.00000.nc"
    with netcdf_file(path, "r", mmap=False) as f:
        assert f.dimensions == {"time": None, "x1": 12, "x1f": 13, "x2": 12, "x2f": 13,
                                "x3": 6, "x3f": 7}
        assert f.variables["x1"].axis == b"Z" and f.variables["x3"].axis == b"X"
        assert f.variables["x2"].long_name == b"Y-coordinate at cell center"
        names = [k for k in f.variables if not k.startswith("x") and k != "time"]
        assert set(names) == {"rho", "press", "vel1", "vel2", "vel3", "H2O", "H2O(l)",
                              "H2O(s)", "temp", "theta"}
        assert f.variables["press"].units == b"pa"
        assert f.variables["theta"].long_name == b"potential temperature"
        assert f.variables["rho"].dimensions == ("time", "x1", "x2", "x3")
        rho = f.variables["rho"][0]
        q = f.variables["H2O"][0]
        np.testing.assert_allclose(f.variables["x1"][:], 125.0 + 250.0 * np.arange(12),
                                   rtol=1e-6)
    w = p.interior(p.w)  # (n, k, j, i)
    assert rho.shape == (12, 12, 6)
    assert np.array_equal(rho, w[0].transpose(2, 1, 0).astype(np.float32))
    assert np.array_equal(q, w[1].transpose(2, 1, 0).astype(np.float32))


def test_theta_of_the_bubble_initial_state():
    p = problems.robert2d(nx1=60, nx2=40)
    f = output.cell_fields(p.cfg, p.w, ("uov",), p.meta["p0"])
    th = f["theta"][:, :, 0]  # (x1, x2)
    x = output.coordinates(p.cfg, p.x1f)
    z, xx = np.meshgrid(x["x1"], x["x2"], indexing="ij")
    r = np.hypot(xx - 500.0, z - 260.0)
    skirt = 0.5 * np.exp(-((r - 50.0) ** 2) / 100.0 ** 2)
    expect = 303.15 + np.where(r <= 50.0, 0.5, skirt)
    np.testing.assert_allclose(th, expect, rtol=0, atol=1e-9)
    assert f["temp"].max() < 303.15 + 0.5


@pytest.mark.parametrize("nb2,nb3", [(2, 2), (4, 1), (1, 2)])
def test_blocks_combine_to_the_domain_file(tmp_path, nb2, nb3):
    p = _c2()
    whole = output.NetcdfOutput(str(tmp_path / "whole"), dt=1.0)
    (ref,) = whole.write(_Block(p, p.w), 3.5)
    o = output.NetcdfOutput(str(tmp_path / "parts"), dt=1.0, keep_blocks=True)
    (got,) = o.write(_Mesh(p, nb2, nb3), 3.5)
    nblk = nb2 * nb3
    for g in range(nblk):
        part = output.block_filename(str(tmp_path / "parts"), g, "out2", 0)
        with netcdf_file(part, "r", mmap=False) as f:
            assert f.NumFilesInSet == nblk
            d2 = f.variables["x2"].domain_decomposition
            d2f = f.variables["x2f"].domain_decomposition
            n2 = 12 // nb2
            o2 = (g % nb2) * n2
            assert list(d2) == [1, 12, o2 + 1, o2 + n2]
            assert list(d2f) == [0, 12, o2, o2 + n2]
    with netcdf_file(ref, "r", mmap=False) as a, netcdf_file(got, "r", mmap=False) as b:
        assert set(a.variables) == set(b.variables)
        for k in a.variables:
            assert np.array_equal(a.variables[k][:], b.variables[k][:]), k
        assert b.variables["theta"].units == b"K"


def _pair(tmp_path, delta):
    p = problems.robert2d(nx1=30, nx2=20)
    a = output.NetcdfOutput(str(tmp_path / "a"), dt=1.0)
    (pa,) = a.write(_Block(p, p.w), 1080.0)
    w = p.w.copy()
    w[4 + p.ny] *= 1.0 + delta  # planted: a pressure error shifts theta
    b = output.NetcdfOutput(str(tmp_path / "b"), dt=1.0)
    (pb,) = b.write(_Block(p, w), 1080.0)
    return pa, pb


def test_regression_check(tmp_path):
    pa, pb = _pair(tmp_path, 0.0)
    assert output.check("robert", pa, pb) == 0.0
    assert output.check("straka", pa, pb) == 0.0
    assert output.main(["robert", pa, pb]) == 0
    # at fixed density theta scales as p^(5/7): 1.5e-3 in p is ~0.32 K per
    # cell, an L2 norm of ~8 over the 600 cells
    pa, pb = _pair(tmp_path, 1.5e-3)
    d = output.l2_difference(pa, pb, "theta", output.CHECKS["robert"][1])
    assert 3.0 < d < 10.0
    assert output.check("robert", pa, pb) == pytest.approx(d)
    pa, pb = _pair(tmp_path, 3e-3)
    with pytest.raises(ValueError, match="robert test failed. L2-norm is"):
        output.check("robert", pa, pb)
    assert output.main(["nope", pa, pb]) == 2


class _Counter:
    """A stepper whose CFL step is fixed: records the steps it takes."""

    def __init__(self, dt):
        self.dt, self.steps = dt, []

    def new_dt(self):
        return self.dt

    def step(self, dt):
        self.steps.append(dt)


class _Recorder:
    def __init__(self, dt):
        self.next_time, self.dt, self.times = 0.0, dt, []

    def due(self, time, tlim, final=False):
        return final or time >= self.next_time or time >= tlim

    def write(self, src, time):
        self.times.append(time)
        self.next_time += self.dt


def test_main_loop_cuts_the_last_step_and_schedules_outputs():
    s = _Counter(0.7)
    o = _Recorder(2.0)
    t, n = driver.evolve(s, 5.0, [o])
    assert t == pytest.approx(5.0) and n == 8
    assert s.steps[:-1] == [0.7] * 7 and s.steps[-1] == pytest.approx(0.1)
    # start, the first cycles at or past 2 and 4, and tlim
    assert o.times == pytest.approx([0.0, 2.1, 4.2, 5.0])
    s2 = _Counter(0.7)
    t, n = driver.evolve(s2, 5.0, nlim=3)
    assert n == 3 and t == pytest.approx(2.1)


@pytest.mark.parametrize("t,name,zmin", [(180.0, "00180s", 300.0), (1080.0, "01080s", 600.0)])
def test_golden_of_the_robert_run(t, name, zmin):
    """The committed oracle outputs of the robert2d run at the first cycle
    past 180 s and at 1080 s (tests/golden/make_robert_golden.py): theta
    only, theta within the initial range (dry adiabatic flow conserves it up
    to the scheme's diffusion) and the bubble risen."""
    path = os.path.join(os.path.dirname(GOLDEN), f"robert2d_ppm.theta.{name}.nc")
    with netcdf_file(path, "r", mmap=False) as f:
        assert abs(float(f.variables["time"][0]) - t) < 0.01
        assert set(f.variables) == {"time", "x1", "x1f", "x2", "x2f", "x3", "theta"}
        th = f.variables["theta"][0, :, :, 0].astype(np.float64)  # (x1, x2)
        z = f.variables["x1"][:].astype(np.float64)
    assert th.shape == (300, 200)
    assert 303.15 - 0.05 < th.min() and th.max() < 303.65 + 0.05
    warm = th > 303.15 + 0.05
    assert warm.any()
    # the warm anomaly's centre of mass has risen above z = 260 m
    zc = float((z[:, None] * (th - 303.15) * warm).sum() / ((th - 303.15) * warm).sum())
    assert zc > zmin


def test_bryan_initial_state():
    """bryan2d: a saturated reversible moist adiabat (theta_e nearly
    constant up the column, liquid everywhere, total water qt) and the
    virtual-temperature bubble of bryan.cpp:125-155 at constant pressure."""
    from canoe_b200 import thermo as T
    p = problems.bryan2d(nx1=50, nx2=100)
    th = p.cfg.thermo
    w = p.interior(p.w)[:, 0]  # (n, j, i)
    q = w[1:3]
    assert np.allclose(q[0] + q[1], 0.0196, rtol=0, atol=1e-12)
    assert (q[1] > 0).all()
    temp = w[4 + th.ny] / (w[0] * th.rd * T.feps_of(th, q))
    te = T.theta_e(th, q, temp, w[4 + th.ny])
    far = te[0]  # the column at x = 100 m, far from the bubble
    assert 319.0 < far.min() and far.max() < 322.0 and far.max() - far.min() < 1.0
    # saturated: the vapour sits at saturation in every cell
    qv, _ = T.sat_split(th, temp, w[4 + th.ny], 0.0196)
    np.testing.assert_allclose(q[0], qv, rtol=1e-9)
    # the bubble: T_v raised by dT cos^2(pi L / 2) T_v / 300 at its centre
    j, i = 50, 9  # x = 10.1 km, z = 1.9 km: L = 0.07
    tv, tv0 = temp[j, i] * T.feps_of(th, q[:, j, i]), temp[0, i] * T.feps_of(th, q[:, 0, i])
    L = np.hypot((10.1e3 - 10.0e3) / 2.0e3, (1.9e3 - 2.0e3) / 2.0e3)
    assert abs(tv / tv0 - (1 + 2.0 * np.cos(np.pi * L / 2) ** 2 / 300.0)) < 1e-9


def test_join_records_and_the_bryan_check(tmp_path):
    p = problems.bryan2d(nx1=20, nx2=40)
    o = output.NetcdfOutput(str(tmp_path / "b"), dt=1.0, variables=("theta_e",))
    for t in range(4):
        o.write(_Block(p, p.w), float(t))
    j = output.join_records(o.written, str(tmp_path / "j.nc"))
    assert list(output.read_variable(j, "time")) == [0.0, 1.0, 2.0, 3.0]
    te = output.read_variable(j, "theta_e")
    assert te.shape == (4, 20, 40, 1)
    assert output.check("bryan", j, j) == 0.0


@pytest.mark.parametrize("name,nrec,t", [("00000-00300s", 4, 300.0), ("01000s", 1, 1000.0)])
def test_golden_of_the_bryan_run(name, nrec, t):
    """The committed oracle outputs of the bryan2d run
    (tests/golden/make_bryan_golden.py): theta_e only, the bubble's theta_e
    above the environment's at the same height, and risen by 1000 s."""
    path = os.path.join(os.path.dirname(GOLDEN), f"bryan2d_ppm.theta_e.{name}.nc")
    with netcdf_file(path, "r", mmap=False) as f:
        assert f.variables["theta_e"].shape == (nrec, 200, 400, 1)
        assert abs(float(f.variables["time"][-1]) - t) < 0.1
        te = f.variables["theta_e"][-1, :, :, 0].astype(np.float64)
    assert 319.0 < te.min() and te.max() < 323.5
    anomaly = te - te[:, :20].mean(axis=1)[:, None]  # against the far columns
    assert anomaly.max() > 1.0
    zmax = np.unravel_index(np.argmax(anomaly), anomaly.shape)[0]
    assert zmax > (60 if t > 500 else 30)  # the bubble started at index 38-40


@pytest.mark.parametrize("name,t", [("00300s", 300.0), ("00900s", 900.0)])
def test_golden_of_the_straka_run(name, t):
    """The committed oracle outputs of the straka2d run
    (tests/golden/make_straka_golden.py): the cold front moving right along
    the ground, at about 15 km by 900 s (Straka et al. 1993 report 14.4 to
    15.5 km across their resolutions)."""
    path = os.path.join(os.path.dirname(GOLDEN), f"straka2d_ppm.theta.{name}.nc")
    with netcdf_file(path, "r", mmap=False) as f:
        assert abs(float(f.variables["time"][0]) - t) < 0.2
        th = f.variables["theta"][0, :, :, 0].astype(np.float64)  # (x1, x2)
        x2 = f.variables["x2"][:].astype(np.float64)
    assert th.shape == (64, 256)
    assert 285.0 < th.min() < 295.0 and th.max() < 300.5
    front = x2[np.where((th < 299.0).any(axis=0))[0].max()]
    assert (3.5e3 < front < 6.0e3) if t < 500 else (14.0e3 < front < 16.0e3)


def test_straka_initial_state():
    """straka.cpp:219-262: the dry adiabat (theta = Ts away from the bubble)
    and the cold bubble, -15 K in temperature (-16.6 K in theta at 3 km) at
    its centre on the left wall."""
    p = problems.straka2d()
    f = output.cell_fields(p.cfg, p.w, ("uov",), p.meta["p0"])
    th = f["theta"][:, :, 0]  # (x1, x2)
    assert np.allclose(th[:, -1], 300.0, rtol=0, atol=1e-9)
    i = 29  # z = 2950 m, x = 50 m: L = 0.027
    assert -17.0 < th[i, 0] - 300.0 < -16.0
